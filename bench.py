"""Throughput of the RHS / RK3 time-advance path on B200.

One step = one full SSPRK3 step (three RHS evaluations, CFL time step,
stage updates, boundary conditions, properties) of the reacting mixing-layer
workload at 256^3 cells (9 species, 19 reactions, MUSCL + AUSM+, laminar,
finite-rate chemistry), FP64. Metric: Mcell-updates/s = cells x steps / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs (torchrun) are independent replicas, one per rank: the
single-GPU path has no exchange step of its own (replicas only); value is
the sum of cell updates over all ranks divided by the max time over ranks.

--impl reference times the CPU implementation of the path: the oracle port
(the reference's kernels restated as FP64 host code, each function citing
the reference file:line it follows; the reference itself runs the path only
as CUDA kernels) with OpenMP on all host cores, on a bounded sample of the
same workload, without loading the product library. The reference's own
CUDA kernels, compiled for sm_100a into oracle/_ref, are timed on the same
workload inside our own line (`reference_cuda_build`).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "openstc-dev_b200"))

FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024  # B200 L2


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixing256",
                    choices=["mixing256", "vortex128", "mixing96", "blocks37", "mixing512"],
                    help="mixing96: the 96^3 mixing layer the kernel profiles are captured on; "
                         "mixing512: the 512x256x256 layer of the learned-chemistry configuration")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-refcuda", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the operator-split comparison (FP64 point-implicit vs learned chemistry)")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the other configurations' legs (small air vortex, 37-block SST RK3 and DPLUR)")
    return ap.parse_args()


def _peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def _make_case(name, full_host=False):
    import ostc

    if name == "mixing256":
        return ostc.case_mixing_layer(256, 256, 256, full_host=full_host)
    if name == "mixing512":
        return ostc.case_mixing_layer(512, 256, 256, full_host=full_host)
    if name == "mixing96":
        return ostc.case_mixing_layer(96, 96, 96, full_host=full_host)
    if name == "blocks37":
        return ostc.case_uneven_blocks(rans_model=2)
    return ostc.case_vortex(128, 128, 8)


def _scheme_text(case, n_blocks=None):
    sc = case.scheme
    rec = {1: "first order", 2: "MUSCL(minmod)", 3: "NND2", 4: "AWENO5"}[sc.reconstruction]
    inv = {1: "L-F", 2: "Roe", 3: "AUSM+", 4: "HLLC"}[sc.inviscid_scheme]
    if sc.reconstruction == 4 and sc.inviscid_scheme == 2:
        inv = "AUSM+"  # quirk A1
    vis = ("k-omega SST" if sc.rans_model == 2 else "laminar") if sc.viscous_order else "inviscid"
    chem = ", finite-rate chemistry" if case.mech is not None else ""
    nb = len(case.blocks) if n_blocks is None else n_blocks
    blocks = ", %d blocks" % nb if nb > 1 else ""
    if sc.steady:
        adv = ("DPLUR (%d sweeps)" % sc.dplur_inner_step if sc.implicit_method == 1 else "explicit") + \
              ", local time stepping CFL %.1f" % sc.cfl
    else:
        adv = "SSPRK3 CFL %.1f" % sc.cfl
    return "%s+%s, %s%s, %s%s" % (rec, inv, vis, chem, adv, blocks)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        if not self.rows:
            return None
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if len(r) > 5 + q and r[5 + q] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# per-kernel timing and the roofline of the dominant kernel
# ---------------------------------------------------------------------------
def kernel_table(solver, case, reps=3):
    """Average device time of each kernel family (CUDA events on the launching
    stream, state left in a valid post-stage condition)."""
    import torch

    ops = [("flux_x", solver.OP_FLUX, 0, 3), ("flux_y", solver.OP_FLUX, 1, 3), ("flux_z", solver.OP_FLUX, 2, 3),
           ("properties", solver.OP_PROPERTIES, 0, 3), ("update_rk", solver.OP_UPDATE, 1, 3),
           ("dt", solver.OP_DT, 0, 3), ("bc", solver.OP_BC, 1, 3)]
    if case.scheme.mix_model == 2 or case.scheme.rans_model == 2:  # chemistry or SST source
        ops.insert(3, ("source", solver.OP_SOURCE, 0, 3))
    out = {}
    for name, op, arg, per_step in ops:
        solver.launch_op(op, arg)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            solver.launch_op(op, arg)
        e1.record()
        torch.cuda.synchronize()
        out[name] = {"ms": e0.elapsed_time(e1) / reps, "per_step": per_step}
    return out


def algorithmic_bytes(name, case):
    """Minimum HBM bytes of one launch of a kernel family on this workload
    (each input plane read once, each output plane written once)."""
    ns = case.mech.n_spec if case.mech else 0
    nt = 2 if case.scheme.rans_model == 2 else 0
    nv = 5 + ns + nt
    cells = case.cells  # one launch covers every block (tile-table launches)
    props = 2 + (ns + 2 if ns else 0) + (3 if nt else 0)  # mu, kappa (+ rho*D_k, cp, gamma) (+ mut, kt, d)
    per_cell = {
        # state (bv 6, sv), geometry (9 metric + jac), properties read; dq read+written
        "flux_x": 6 + ns + nt + 10 + props + 2 * nv,
        "flux_y": 6 + ns + nt + 10 + props + 2 * nv,
        "flux_z": 6 + ns + nt + 10 + props + 2 * nv,
        "source": (2 + ns + 1 + nv) if not nt else (6 + nt + 10 + 1 + 1 + nv + 2),
        "properties": 6 + ns + 1 + props + 3,
        "update_rk": 3 * nv + 1 + nv + 6 + ns + nt + 1,
        "dt": 9 + 6 + 3,
        "bc": 0,
    }[name]
    return 8.0 * per_cell * cells


# ---------------------------------------------------------------------------
# replicas (one independent copy of the workload per rank; no collective on
# the data path): the job ends with its slowest rank
# ---------------------------------------------------------------------------
def replica_ms(ms, world, device):
    """the device-timed ms of this rank -> the max over all ranks"""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cells, steps, world, ms):
    """whole-job Mcell-updates/s: every rank advanced its own cells"""
    return cells * steps * world / (ms * 1e-3) / 1e6


# ---------------------------------------------------------------------------
# the timed run
# ---------------------------------------------------------------------------
def run_ours(a):
    import numpy as np
    import torch
    import torch.distributed as dist

    import ostc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    case = _make_case(a.workload)
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    solver = ostc.Solver(case.scheme, case.mech, blocks, case.faces, interfaces=case.interfaces)
    solver.initialize()
    solver.autotune(warmup=1, reps=2)
    solver.initialize()  # autotuning ran RHS evaluations only; re-derive the same start state
    torch.cuda.synchronize()
    solver.rk3_steps(max(a.warmup, 3))
    torch.cuda.synchronize()
    launches_per_step = solver.step_kernel_count(False)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    small = state_bytes(case) < 2 * L2_BYTES
    if small:
        # a state that fits in L2: every step timed on its own after a write of 2x L2 that evicts it
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
        ms_dev = 0.0
        for _ in range(a.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            solver.rk3_steps(1)
            e1.record()
            torch.cuda.synchronize()
            ms_dev += e0.elapsed_time(e1)
        del flush
    else:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.rk3_steps(a.steps)
        e1.record()
        torch.cuda.synchronize()
        ms_dev = e0.elapsed_time(e1)
    if world > 1:
        dist.barrier()
    ck = clocks.stop()
    ms = replica_ms(ms_dev, world, "cuda")
    cells = case.cells
    value = replica_value(cells, a.steps, world, ms)

    # several blocks: the same steps with one launch per block instead of the
    # tile-table launches (same tiles, same start state)
    per_block = None
    if len(case.blocks) > 1:
        solver.initialize()
        solver.set_batching(False)
        solver.rk3_steps(max(a.warmup, 3))
        torch.cuda.synchronize()
        lpb = solver.step_kernel_count(False)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        solver.rk3_steps(a.steps)
        p1.record()
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        per_block = {"value": round(case.cells * a.steps / (pms * 1e-3) / 1e6, 2), "unit": "Mcell-updates/s",
                     "ms_per_step": round(pms / a.steps, 4), "launches_per_step": lpb,
                     "tile_table_speedup": round(pms / ms, 3)}
        solver.set_batching(True)
        solver.initialize()
        solver.rk3_steps(1)
        torch.cuda.synchronize()

    # per-kernel table and roofline of the dominant kernel (the family with the
    # largest share of the step; the three flux directions are one kernel template)
    ktab = kernel_table(solver, case)
    families = {"flux": ["flux_x", "flux_y", "flux_z"]}
    for k in ktab:
        if not k.startswith("flux_"):
            families[k] = [k]
    share = {f: sum(ktab[k]["ms"] * ktab[k]["per_step"] for k in ks) for f, ks in families.items()}
    dom = max(share, key=share.get)
    ks = families[dom]
    hbm, src = _peaks()
    alg = sum(algorithmic_bytes(k, case) for k in ks) / len(ks)
    launch_ms = sum(ktab[k]["ms"] for k in ks) / len(ks)
    achieved = alg / (launch_ms * 1e-3) / 1e9
    traffic = None
    tf = REPO / "profiles" / "traffic.json"
    if tf.exists():
        try:
            tt = json.loads(tf.read_text()).get(a.workload, {}).get(dom)
            traffic = float(tt) if tt is not None else None
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_source": src, "traffic": traffic,
                "alg_bytes_per_launch": alg, "launch_ms": round(launch_ms, 4),
                "step_share": round(share[dom] / sum(share.values()), 3)}
    # whole-step roofline: minimum Field traffic of one cell through one RK3 step
    b_alg = step_bytes_per_cell(case)
    step_roofline = {"bytes_per_cell_update": b_alg, "achieved": round(value * 1e6 * b_alg / 1e9, 1),
                     "peak": hbm, "unit": "GB/s", "frac": round(value * 1e6 * b_alg / 1e9 / hbm, 4)}

    # end to end through the public API from host buffers
    tiles = solver.tiles()
    solver.close()
    del blocks
    torch.cuda.empty_cache()
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, case, tiles)

    legs = None
    if rank == 0 and world == 1 and not a.no_legs and a.workload == "mixing256":
        legs = {}
        for key, w, st in (("C1_vortex_128x128x8", "vortex128", False), ("C3_blocks37_sst_rk3", "blocks37", False),
                           ("C3_blocks37_sst_dplur", "blocks37", True)):
            try:
                legs[key] = run_config_leg(a, w, steady=st)
            except Exception as exc:  # reported, not fatal for the headline line
                legs[key] = {"error": repr(exc)[:300]}
    surr = None
    if rank == 0 and world == 1 and not a.no_surrogate and case.mech is not None:
        try:
            # the learned-chemistry configuration: the layer at 512 x 256 x 256
            surr = run_surrogate_compare(a, tiles, "mixing512" if a.workload == "mixing256" else None)
        except Exception as exc:  # reported, not fatal for the headline line
            surr = {"error": repr(exc)[:300]}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_baseline(a)
    refcuda = None
    if rank == 0 and world == 1 and not a.no_refcuda:
        refcuda = reference_cuda_build(a, value)

    if rank == 0:
        line = {"metric": "Mcell-updates/s per RK3 step (plain FP64 chemistry)", "value": round(value, 2),
                "unit": "Mcell-updates/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(a, world, case),
                "gpu_launches": launches_per_step * a.steps, "launches_per_step": launches_per_step,
                "tiles": tiles,
                "clocks": ck, "roofline": roofline, "step_roofline": step_roofline, "kernels_ms": {k: round(v["ms"], 4) for k, v in ktab.items()},
                "e2e": e2e, "cpu_baseline": cpu, "reference_cuda_build": refcuda, "surrogate_chem": surr,
                "other_configs": legs}
        if per_block is not None:
            line["per_block_launches"] = per_block
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def _timed_steps(solver, steps, small, steady=False):
    """device ms of `steps` steps: each step timed alone after a 2x L2 write
    when the state is smaller than 2x L2, else all steps back to back"""
    import torch

    go = (lambda n: solver.steady_steps(n)) if steady else (lambda n: solver.rk3_steps(n))
    if small:
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
        ms = 0.0
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            go(1)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    go(steps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_config_leg(a, workload, steady=False):
    """One more configuration on the same GPU, through the same API: its own
    workload, autotuned tiles, W warm-up and K timed steps (RK3 steps, or
    DPLUR steady iterations with 3 inner sweeps), with its step roofline."""
    import torch

    import ostc

    case = _make_case(workload)
    if steady:
        case = ostc.make_steady(case, implicit_method=1, dplur_inner_step=3)
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    solver = ostc.Solver(case.scheme, case.mech, blocks, case.faces, interfaces=case.interfaces)
    solver.initialize()
    if not steady:
        solver.autotune(warmup=1, reps=2)
        solver.initialize()
    torch.cuda.synchronize()
    (solver.steady_steps if steady else solver.rk3_steps)(max(a.warmup, 3))
    torch.cuda.synchronize()
    small = state_bytes(case) < 2 * L2_BYTES
    steps = min(a.steps, 20)
    ms = _timed_steps(solver, steps, small, steady)
    hbm, src = _peaks()
    value = case.cells * steps / (ms * 1e-3) / 1e6
    out = {"workload": case.name, "cells": case.cells, "scheme": _scheme_text(case), "steps": steps,
           "value": round(value, 2), "unit": "Mcell-updates/s", "ms_per_step": round(ms / steps, 4),
           "launches_per_step": solver.step_kernel_count(False),
           "l2": "flushed before each step" if small else "inputs larger than L2"}
    if steady:
        out["iterations_per_s"] = round(steps / (ms * 1e-3), 2)
        out["method"] = "DPLUR, 3 inner sweeps, local time stepping"
    else:
        b_alg = step_bytes_per_cell(case)
        out["step_roofline"] = {"bytes_per_cell_update": b_alg, "achieved": round(value * 1e6 * b_alg / 1e9, 1),
                                "peak": hbm, "unit": "GB/s", "frac": round(value * 1e6 * b_alg / 1e9 / hbm, 4),
                                "peak_source": src}
        ktab = kernel_table(solver, case)
        out["kernels_ms"] = {k: round(v["ms"], 4) for k, v in ktab.items()}
        fl = [k for k in ktab if k.startswith("flux_")]
        alg = sum(algorithmic_bytes(k, case) for k in fl) / len(fl)
        lm = sum(ktab[k]["ms"] for k in fl) / len(fl)
        out["flux_roofline"] = {"achieved": round(alg / (lm * 1e-3) / 1e9, 1), "peak": hbm, "unit": "GB/s",
                                "frac": round(alg / (lm * 1e-3) / 1e9 / hbm, 4), "launch_ms": round(lm, 4)}
    solver.close()
    del blocks
    torch.cuda.empty_cache()
    return out


def run_surrogate_compare(a, tiles, workload=None):
    """Plain vs learned chemistry on the same workload, both operator-split
    (the flow's three RK3 stages, then each cell's chemistry over the step's
    dt): chem_mode 1 runs the FP64 point-implicit integrator, chem_mode 2 the
    tcgen05 surrogate with FP64 fallback. The surrogate is first trained
    (timed separately) on 4M labelled states: 2M sampled from snapshots of
    FP64 operator-split runs of 64 x 256 x 64 slabs of the layer (its full y
    extent) with other noise seeds
    (surrogate.trajectory_states) and 2M from the synthetic sampler over the
    training envelope, so the evaluated workload is held out. Both runs
    start from the same state; the final fields are compared after warm-up
    + timed steps. The chemistry operator alone (the learned step with its
    fallback against the FP64 integrator, on the cells of the final field
    at the step's dt) is timed as well."""
    import numpy as np
    import torch

    import ostc
    import surrogate as S

    workload = workload or a.workload
    lab_case = ostc.case_premixed_box(8, 8, 4)
    lab_solver, _ = lab_case.solver()
    mech = lab_case.mech
    torch.cuda.synchronize()
    t0 = time.time()
    # slabs of the layer with its full 256-cell y extent, so the pure streams
    # (no fuel on the air side, no oxygen on the fuel side) are in the data
    traj = S.trajectory_states(2_000_000, size=(64, 256, 64), seeds=(5, 6), steps=40, every=10, seed=17)
    sur, sc, log = S.build(lab_solver, mech, n_train=2_000_000, epochs=20, seed=1, extra_states=traj)
    torch.cuda.synchronize()
    train_s = time.time() - t0
    n_samples = log.steps * 65536
    out = {"train": {"states": 4_000_000, "epochs": 20, "batch": 65536, "steps": log.steps,
                     "train_seconds": round(log.seconds, 3), "pipeline_seconds": round(train_s, 3),
                     "samples_per_s": round(n_samples / log.seconds, 1),
                     "tflops": round(3 * 273408 * n_samples / log.seconds / 1e12, 2),
                     "final_loss": log.loss[-1]}}
    finals, rates = {}, {}
    for mode in (1, 2):
        c = _make_case(workload)
        c.scheme.chem_mode = mode
        s, blocks = c.solver()
        s.set_tiles(tiles)
        if mode == 2:
            s.set_chem_surrogate(sur)
        s.initialize()
        s.rk3_steps(max(a.warmup, 3))
        n0, f0 = s.chem_stats()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.rk3_steps(a.steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        n1, f1 = s.chem_stats()
        rates[mode] = {"value": round(c.cells * a.steps / (ms * 1e-3) / 1e6, 2), "ms_per_step": round(ms / a.steps, 3),
                       "fallback_fraction": round((f1 - f0) / max(1, n1 - n0), 5)}
        finals[mode] = (blocks[0].t["bv"][5].clone(), blocks[0].t["sv"].clone())
        if mode == 2:
            # the chemistry operator alone on the cells of the final field at the last dt
            g = c.blocks[0].ngg
            bvt, svt = blocks[0].t["bv"], blocks[0].t["sv"]
            st = [bvt[5, g:-g, g:-g, g:-g].reshape(-1).contiguous(), bvt[4, g:-g, g:-g, g:-g].reshape(-1).contiguous(),
                  svt[:, g:-g, g:-g, g:-g].reshape(svt.shape[0], -1).contiguous()]
            _, dts = s.rk3_steps(1, history=True)
            st.append(torch.full_like(st[0], float(dts[-1])))
            lab_solver.chem_surrogate(sur, *st)
            lab_solver.chem_point_implicit(*st)
            t_ops = {}
            for nm, fn in (("surrogate", lambda: lab_solver.chem_surrogate(sur, *st)),
                           ("fp64_integrator", lambda: lab_solver.chem_point_implicit(*st))):
                torch.cuda.synchronize()
                q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                q0.record()
                for _ in range(3):
                    r = fn()
                q1.record()
                torch.cuda.synchronize()
                t_ops[nm] = q0.elapsed_time(q1) / 3
            nfb = lab_solver.chem_surrogate(sur, *st)[2]
            chem_op = {"states": st[0].numel(), "ms_surrogate": round(t_ops["surrogate"], 3),
                       "ms_fp64_integrator": round(t_ops["fp64_integrator"], 3),
                       "ns_per_state_surrogate": round(t_ops["surrogate"] * 1e6 / st[0].numel(), 3),
                       "ns_per_state_integrator": round(t_ops["fp64_integrator"] * 1e6 / st[0].numel(), 3),
                       "speedup": round(t_ops["fp64_integrator"] / t_ops["surrogate"], 3),
                       "fallback_fraction": round(nfb / st[0].numel(), 5),
                       "tensor_tflops": round(273408 * st[0].numel() / (t_ops["surrogate"] * 1e-3) / 1e12, 1)}
            del st
        s.close()
        del blocks
        torch.cuda.empty_cache()
    dT = (finals[2][0] - finals[1][0]).abs()
    dY = (finals[2][1] - finals[1][1]).abs()
    out.update({"workload": _make_case_name(workload), "chemistry_operator": chem_op,
                "unit": "Mcell-updates/s", "plain_split_fp64": rates[1], "surrogate_split": rates[2],
                "speedup_surrogate_over_plain_split": round(rates[2]["value"] / rates[1]["value"], 3),
                "final_field_vs_plain": {"steps": max(a.warmup, 3) + a.steps, "max_abs_dT_K": float(dT.max()),
                                         "mean_abs_dT_K": float(dT.mean()), "max_abs_dY": float(dY.max()),
                                         "mean_abs_dY": float(dY.mean())}})
    sur.close()
    lab_solver.close()
    return out


def step_bytes_per_cell(case):
    """B_alg of one cell through one RK3 step: per stage the state (bv 6,
    sv) and geometry (9 metric + jac) read and bv, sv, cv written; stages 2-3
    read u^n. Derived properties are recomputed, not counted."""
    ns = case.mech.n_spec if case.mech else 0
    nt = 2 if case.scheme.rans_model == 2 else 0  # SST: k, omega and the wall distance
    nsc, nv, geo = ns + nt, 5 + ns + nt, 10 + (1 if nt else 0)
    return 8 * (3 * (6 + nsc + geo) + 2 * nv + 3 * (6 + nsc + nv))


def state_bytes(case):
    return state_bytes_dims(case, [(b.mx, b.my, b.mz) for b in case.blocks], case.blocks[0].ngg)


def state_bytes_dims(case, dims, ngg):
    ns = case.mech.n_spec if case.mech else 0
    nt = 2 if case.scheme.rans_model == 2 else 0
    return sum(8.0 * (6 + ns + nt + 10 + 2 * (5 + ns + nt)) * (x + 2 * ngg) * (y + 2 * ngg) * (z + 2 * ngg)
               for x, y, z in dims)


def run_e2e(a, case, tiles=None):
    """Whole job through the public API from pinned host buffers: upload of the
    initial state and geometry, initialisation, the steps, download of the
    final primitive state and the residual history; timed with CUDA events."""
    import numpy as np
    import torch

    import ostc

    pinned = [{n: torch.from_numpy(v.view(np.uint8).reshape(-1) if n == "metric" else v).pin_memory()
               for n, v in host.arrays.items()} for host in case.blocks]
    blocks = [ostc.DeviceBlock(ostc.HostBlock(h.mx, h.my, h.mz, h.ngg, h.n_var, h.n_spec, n_turb=h.n_turb))
              for h in case.blocks]
    out_bv = [torch.empty_like(b.t["bv"], device="cpu").pin_memory() for b in blocks]
    out_sv = [torch.empty_like(b.t["sv"], device="cpu").pin_memory() for b in blocks]
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    h2d = 0
    for b, pin in zip(blocks, pinned):
        for n, t in pin.items():
            b.t[n].copy_(t.view(b.t[n].dtype).reshape(b.t[n].shape), non_blocking=True)
            h2d += t.numel() * t.element_size()
    solver = ostc.Solver(case.scheme, case.mech, blocks, case.faces, interfaces=case.interfaces)
    solver.set_tiles(tiles)
    solver.initialize()
    res, dts = solver.rk3_steps(a.steps, history=True)
    for b, ob, os_ in zip(blocks, out_bv, out_sv):
        ob.copy_(b.t["bv"], non_blocking=True)
        os_.copy_(b.t["sv"], non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    d2h = sum(t.numel() * 8 for t in out_bv + out_sv) + res.size * 8 + dts.size * 8
    solver.close()
    assert np.all(np.isfinite(res)), "non-finite residual in the e2e run"
    return {"value": round(case.cells * a.steps / (ms * 1e-3) / 1e6, 2), "unit": "Mcell-updates/s",
            "h2d_bytes_per_step": int(h2d / a.steps), "d2h_bytes_per_step": int(d2h / a.steps),
            "ms_total": round(ms, 2), "includes": "H2D state+geometry, initialize, steps, D2H bv/sv/residuals"}


# ---------------------------------------------------------------------------
# CPU legs (the oracle port on the host cores) and the reference's CUDA build
# ---------------------------------------------------------------------------
def _cpu_case(w):
    """The bounded CPU sample of workload w and its description. The mixing
    layers are sampled by a 256 x 256 x 8 slab of the same layer (same x-y
    extent, tanh profiles, stream states and noise distribution; z periodic
    as in the full case), so the per-cell work is the full case's."""
    import ostc

    if w in ("mixing256", "mixing512", "mixing96"):
        nx = {"mixing256": 256, "mixing512": 512, "mixing96": 96}[w]
        ny = 96 if w == "mixing96" else 256
        case = ostc.case_mixing_layer(nx, ny, 8, full_host=True)
        return case, "%dx%dx8 slab of the layer (%d cells)" % (nx, ny, case.cells)
    if w == "blocks37":
        case = ostc.case_uneven_blocks(layout=ostc.block_layout(5, dims=(80, 64, 64), ranges=((16, 40), (16, 28),
                                                                                              (16, 20)),
                                                                anchors=False), rans_model=2)
        return case, "5 uneven SST blocks (%d cells) of the same scheme" % case.cells
    case = ostc.case_vortex(128, 128, 8)
    return case, "the whole 128x128x8 case"


def cpu_sample(a, budget_s=15.0, max_steps=50):
    """Time the oracle port (the CPU restatement of the reference's path,
    OpenMP over all host cores) on the bounded sample of the workload,
    stepping RK3 until ~budget_s."""
    sys.path.insert(0, str(REPO / "tests"))
    from oracle_bind import OracleRun

    case, what = _cpu_case(a.workload)
    r = OracleRun(case)
    r.initialize()
    steps, t0 = 0, time.perf_counter()
    while True:
        r.rk3_steps(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= max_steps:
            break
    value = case.cells * steps / el / 1e6
    return {"value": round(value, 4), "unit": "Mcell-updates/s", "cores": r.threads(), "kind": "port",
            "sample": "%s, %d RK3 steps, %.1f s" % (what, steps, el)}


def cpu_baseline(a):
    return cpu_sample(a)


def reference_cuda_build(a, ours_value):
    """The reference's own kernels (sources compiled for sm_100a, driven by
    oracle/ref_cuda_harness.cu through RK3_bv's per-step sequence) on the same
    workload, timed with CUDA events: 10 warm-up steps, then the median of 3
    runs of 5 steps. Periodic faces become extrapolation faces since the
    reference has no periodic boundary."""
    sys.path.insert(0, str(REPO / "tests"))
    import ref_bind

    if not ref_bind.available():
        return {"unavailable": "oracle/_ref/libostc_ref_cuda.so not built (needs the reference sources)"}
    import ostc

    case = _make_case(a.workload)
    for f in case.faces:
        # no periodic boundary in the reference; its air + SST far field reads
        # unset boundary scalars on subsonic outflow: both become outflow faces
        if f.type_label == ostc.BC_PERIODIC or (case.scheme.rans_model and f.type_label == ostc.BC_FARFIELD):
            f.type_label = ostc.BC_OUTFLOW
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    r.time_steps(10)
    n, runs = 5, []
    for _ in range(3):
        runs.append(r.time_steps(n) / n)
    ms = sorted(runs)[1]
    v = case.cells / (ms * 1e-3) / 1e6
    return {"value": round(v, 2), "unit": "Mcell-updates/s", "ms_per_step": round(ms, 3),
            "protocol": "10 warm-up steps, median of 3 runs of 5 steps (CUDA events)",
            "runs_ms_per_step": [round(x, 3) for x in runs],
            "speedup_ours_over_reference_build": round(ours_value / v, 2),
            "note": "reference sources compiled for sm_100a, same workload, extrapolation faces instead of periodic"
                    " (and of the SST far field)"}


def workload_config(a, world, case=None, sample=None):
    """The `config` object of a bench line: the same for both arms (the
    reference arm describes the workload from its bounded sample without
    building it at full size)."""
    if case is None:
        small = sample if sample is not None else _cpu_case(a.workload)[0]
        if a.workload == "blocks37":
            small = _make_case(a.workload)
        dims = {"mixing256": [(256, 256, 256)], "mixing512": [(512, 256, 256)], "mixing96": [(96, 96, 96)],
                "vortex128": [(128, 128, 8)]}.get(a.workload, [(b.mx, b.my, b.mz) for b in small.blocks])
        ng = small.blocks[0].ngg
        info = dict(name=_make_case_name(a.workload), mech=small.mech, scheme_case=small,
                    cells=sum(x * y * z for x, y, z in dims), dims=dims, ngg=ng)
    else:
        info = dict(name=case.name, mech=case.mech, scheme_case=case, cells=case.cells,
                    dims=[(b.mx, b.my, b.mz) for b in case.blocks], ngg=case.blocks[0].ngg)
    sb = state_bytes_dims(info["scheme_case"], info["dims"], info["ngg"])
    small_state = sb < 2 * L2_BYTES
    return {"workload": info["name"], "cells_per_gpu": info["cells"],
            "n_spec": info["mech"].n_spec if info["mech"] else 0,
            "n_reac": info["mech"].n_reac if info["mech"] else 0,
            "scheme": _scheme_text(info["scheme_case"], n_blocks=len(info["dims"])),
            "parallelism": "replicas" if world > 1 else "single",
            "l2": ("state %.2f GB below 2x L2: L2 flushed (%d MB written) before each step, steps timed one by "
                   "one" % (sb / 1e9, 2 * L2_BYTES >> 20)) if small_state else
                  "inputs larger than L2 (%.1f GB state), no flush" % (sb / 1e9)}


def _libostc_mapped():
    try:
        return any("libostc.so" in ln for ln in open("/proc/self/maps"))
    except OSError:
        return False


def run_reference(a):
    """The reference arm: the CPU implementation of the path (the oracle
    port, a cited FP64 restatement of the reference's kernels; the reference
    itself has no CPU code) on all host cores. Each timed step is one RK3
    step of the bounded sample of the workload. The product library is never
    loaded: the workloads' geometry comes from the numpy restatement of the
    reference's metric (oracle/metric_oracle.py)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sys.path.insert(0, str(REPO / "oracle"))
    sys.path.insert(0, str(REPO / "tests"))
    import metric_oracle
    import ostc
    from oracle_bind import OracleRun

    ostc.set_metric_provider(metric_oracle.metric)
    case, what = _cpu_case(a.workload)
    r = OracleRun(case)
    r.initialize()
    for _ in range(a.warmup):
        r.rk3_steps(1)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        r.rk3_steps(1)
    el = time.perf_counter() - t0
    value = round(case.cells * a.steps / el / 1e6, 4)
    sample = "%s, %d timed RK3 steps after %d warm-up, %.1f s" % (what, a.steps, a.warmup, el)
    assert not _libostc_mapped(), "the reference arm must not load the product library"
    line = {"impl": "reference", "metric": "Mcell-updates/s per RK3 step (plain FP64 chemistry)", "value": value,
            "unit": "Mcell-updates/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(el * 1e3 / a.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a, world, sample=case),
            "sample": sample,
            "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": r.threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _make_case_name(w):
    return {"mixing256": "mixing_layer_h2air_256x256x256", "mixing96": "mixing_layer_h2air_96x96x96",
            "mixing512": "mixing_layer_h2air_512x256x256",
            "blocks37": "uneven_blocks_37_air_sst_10453312cells"}.get(w, "vortex_air_128x128x8")


if __name__ == "__main__":
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
