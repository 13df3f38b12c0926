"""Benchmark of the GSO docking step on B200 (scored poses/s and GSO steps/s).

One bench step = one GSO step over every glowworm of the workload (rescore moved poses,
luciferin, neighbour selection, movement).  Default workload: the mixed-precision batched step,
eight synthetic complexes of uneven sizes (757/481 ... 6143/633 atoms, 130 ... 695 swarms x 200
glowworms, 640,400 poses, 10+10 ANM modes) in one persistent scorer launch per step, replayed
from a CUDA graph; 3 warm-up steps + 97 timed steps = the workload's 100 GSO steps.  The plain
FP64 kernels run the same steps from the same start for the mixed-vs-FP64 ratio.  The same line
carries the single complex (3002 / 1274 atoms, 402 x 200 glowworms) under "c1", with its own
ratio and a per-step check of its energies against the plain FP64 kernel.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c2]

--impl reference: the reference's own CPU path (compiled from its sources into oracle/_ref) on a
bounded sample of the same workload, with inputs from the oracle; the product library is not
loaded in that process.

N > 1 (torchrun): every rank runs its own replica of the workload on its GPU (the swarms of
the reference shard with no data exchange); value = all ranks' scored poses / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c0": dict(workload="single complex, plain FP64", complexes=[(757, 481, 130)], precision="fp64", steps=100),
    "c1": dict(workload="single complex, mixed precision", complexes=[(3002, 1274, 402)], precision="mixed",
               steps=100),
    "c2": dict(workload="8 complexes batched, mixed precision",
               complexes=[(757, 481, 130), (2039, 1440, 271), (2516, 1061, 298), (2030, 1256, 294),
                          (3052, 1658, 336), (6058, 1138, 558), (6032, 1766, 695), (6143, 633, 620)],
               precision="mixed", steps=100, cmp_steps=4),
    "c3": dict(workload="large receptor, mixed precision", complexes=[(17307, 1125, 1245)], precision="mixed",
               steps=50, cmp_steps=4),
    "c4": dict(workload="pyDock-style energy adjoint (4096 poses) + refinement of the top 5 per swarm",
               complexes=[(3002, 1274, 402)], precision="mixed", steps=100),
}
G = 200
METRIC = "scored poses/s and GSO steps/s on 1 B200, mixed vs FP64 at <=1e-5 rel energy err"
L2_FLUSH_BYTES = 256 << 20
# DRAM traffic of one mixed DFIRE scorer launch after the L2 flush, from ncu
# dram__bytes_read.sum + dram__bytes_write.sum of three launches (4,098 / 5,658 / 6,483 poses
# rescored) on the 3002 / 1274-atom complex with 40 swarms: a fixed part (the L2-resident tables
# and atom arrays read once per launch) plus a part per rescored pose (pose in, score and
# reference point out), a least-squares fit, as summarised with the scorer's launch list under profiles/
DRAM_BYTES_PER_LAUNCH = 9.12e6
DRAM_BYTES_PER_SCORED_POSE = 212.0
# warp-instructions the mixed scorer issues per receptor-ligand pair inside the cutoff, from ncu
# smsp__inst_executed.sum of one launch (3002 / 1274 atoms, 4,098 poses, 233.9 M pairs in the
# cutoff), as summarised with its full capture under profiles/; one ceiling of the scorer is the
# SMs' issue rate (148 SMs x 4 schedulers x clock) over this count
WARP_INSTR_PER_PAIR = 5.96
# L1 data-pipe wavefronts per in-cutoff pair in the same launch (l1tex__data_pipe_lsu_wavefronts:
# 228.5 M shared-memory wavefronts plus ~181.6 M global-load ones, nearly all table gathers, over
# 233.9 M pairs); the pipe retires one wavefront per SM per cycle, the other ceiling
L1_WAVEFRONTS_PER_PAIR = 1.75


def make_complexes(cfg, seed0=100):
    import sparkledock_b200 as sd
    return [sd.SyntheticComplex(nr, nl, s, G, 10, 10, seed=seed0 + i) for i, (nr, nl, s) in enumerate(cfg["complexes"])]


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def brute_pairs_per_pose(cfg):
    """Receptor x ligand atom pairs of one pose, averaged over the poses of every complex (each
    complex weighted by its swarm count: all glowworms of a step are candidates for rescoring)."""
    cs = cfg["complexes"]
    return sum(nr * nl * s for nr, nl, s in cs) / sum(s for _, _, s in cs)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def run_gpu(cfg, prec_name, steps, warmup, device, flush, seed=0, per_step=False, energy_every=0):
    """Device-timed run: draws resident in HBM, per-step CUDA events on the context stream,
    L2 flushed (256 MB write) between timed steps outside the events.  energy_every = k > 0:
    after every k-th timed step (outside the events) the scores that step wrote for the poses it
    rescored are checked against the plain FP64 kernel on the same poses (up to 256 per complex)."""
    import torch
    import sparkledock_b200 as sd
    prec = {"mixed": sd.SD_PREC_MIXED, "fp64": sd.SD_PREC_FP64, "fp64_ref": sd.SD_PREC_FP64_REF}[prec_name]
    cxs = make_complexes(cfg)
    tables = sd.synthetic_tables(3)
    total = warmup + steps
    dk = sd.Docking(cxs, tables, precision=prec, device=device)
    for i, c in enumerate(cxs):
        dk.init_state(i, c.poses)
        dk.set_draws(i, sd.gso_draws(seed + i, c.n_swarms, total, c.n_glowworms))
    stream = torch.cuda.ExternalStream(dk.stream, device=device)
    dk.step(warmup, sync=True)
    s0 = dk.stats()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    scored_steps = []
    pair_steps = []
    energy_err = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            check = energy_every > 0 and k % energy_every == 0
            before = [dk.get_state(i) for i in range(len(cxs))] if check else None
            if flush is not None:
                flush.zero_()
            starts[k].record(stream)
            dk.step(1, sync=False)
            ends[k].record(stream)
            if per_step:  # synchronises between steps (outside the timed events)
                st = dk.stats()
                scored_steps.append(st["scored_poses"])
                pair_steps.append(st["pairs_in_cutoff"])
            if check:
                energy_err.append(step_energy_error(dk, cxs, before, k))
    torch.cuda.synchronize(device)
    ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    s1 = dk.stats()
    out = {"ms": ms, "scored": s1["scored_poses"] - s0["scored_poses"], "stats": s1, "ctx": dk, "cxs": cxs,
           "pairs": s1["pairs_in_cutoff"] - s0["pairs_in_cutoff"],
           "tuning": dk.tuning(),
           "per_step": [b - a for a, b in zip([s0["scored_poses"]] + scored_steps, scored_steps)] if per_step else None,
           "per_step_pairs": ([b - a for a, b in zip([s0["pairs_in_cutoff"]] + pair_steps, pair_steps)]
                              if per_step else None),
           "energy_err": energy_err}
    return out


def step_energy_error(dk, cxs, before, k, per_complex=256):
    """Scores written by one GSO step for the poses it rescored (moved in the step before, or not
    yet scored), against the plain FP64 kernel on the same poses (the pose each had when the
    step began): max |s_mixed - s_fp64| / max(|s_fp64|, 1) and the same on the raw DFIRE energy
    E = (4.7 - s) / 0.0157."""
    import sparkledock_b200 as sd
    worst_s, worst_e, n = 0.0, 0.0, 0
    for i, c in enumerate(cxs):
        b = before[i]
        sel = np.flatnonzero(((b.moved == 1) | (b.step == 0)).ravel())
        if sel.size == 0:
            continue
        sel = sel[np.linspace(0, sel.size - 1, min(per_complex, sel.size)).astype(int)]
        after = dk.get_state(i).scoring.ravel()[sel]
        s64, e64 = dk.score_poses(i, b.pos.reshape(-1, c.pose_len)[sel], sd.SD_PREC_FP64)
        worst_s = max(worst_s, float((np.abs(after - s64) / np.maximum(np.abs(s64), 1.0)).max()))
        e_mixed = (4.7 - after) / 0.0157
        worst_e = max(worst_e, float((np.abs(e_mixed - e64) / np.maximum(np.abs(e64), 1.0)).max()))
        n += sel.size
    return {"step": k, "poses": n, "max_rel_score_err": worst_s, "max_rel_energy_err": worst_e}


def time_clustering(dk, cxs):
    """Wall clock of one sd_cluster call on the final poses of the first complex (every swarm),
    backbone = every 8th atom (about one CA per residue of a protein)."""
    c = cxs[0]
    rb = (np.arange(c.n_rec) % 8 == 1).astype(np.int32)
    lb = (np.arange(c.n_lig) % 8 == 1).astype(np.int32)
    dk.cluster(0, rb, lb)
    t0 = time.perf_counter()
    out = dk.cluster(0, rb, lb)
    dt = time.perf_counter() - t0
    return {"ms": dt * 1e3, "swarms": c.n_swarms, "glowworms": c.n_glowworms,
            "backbone_atoms": int(rb.sum() + lb.sum()), "mean_clusters_per_swarm": float(out["n_clusters"].mean())}


def fp64_spot_check(dk, cxs, frac=0.01):
    """Energies of 1 % of the final poses (at least 256 per complex) from the mixed kernel
    against the plain FP64 kernel: max |E_mixed - E_fp64| / max(|E_fp64|, 1) on the raw DFIRE
    sum, and the same on the score (the reference's `energy`, -(0.0157 E - 4.7))."""
    import sparkledock_b200 as sd
    worst, worst_sc, n = 0.0, 0.0, 0
    for i, c in enumerate(cxs):
        pos = dk.get_state(i).pos.reshape(-1, c.pose_len)
        k = max(256, int(frac * len(pos)))
        sel = pos[np.linspace(0, len(pos) - 1, min(k, len(pos))).astype(int)]
        s32, e32 = dk.score_poses(i, sel, sd.SD_PREC_MIXED)
        s64, e64 = dk.score_poses(i, sel, sd.SD_PREC_FP64)
        worst = max(worst, float((np.abs(e32 - e64) / np.maximum(np.abs(e64), 1.0)).max()))
        worst_sc = max(worst_sc, float((np.abs(s32 - s64) / np.maximum(np.abs(s64), 1.0)).max()))
        n += len(sel)
    return {"poses": n, "max_rel_energy_err": worst, "max_rel_score_err": worst_sc, "tolerance": 1e-5}


def run_c4(cfg, device, gso_steps, steps, warmup, flush, refine_iters=50):
    """Adjoint throughput and accuracy on 4096 poses, then refinement of the top 5 glowworms per
    swarm after a DFIRE GSO run, judged by the FP64 pyDock-style energy.  A step is one
    sd_pydock_grad call over the 4096 poses: host buffers in (poses) and out (energies,
    gradients), synchronous, so each call is timed by the wall clock around it, with the L2
    flushed before it; warm-up calls first (the first one sizes the context's scratch)."""
    import torch
    import sparkledock_b200 as sd
    nr, nl, S = cfg["complexes"][0]
    cx = sd.SyntheticComplex(nr, nl, S, G, 10, 10, seed=100)
    tables = sd.synthetic_tables(3)
    poses = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len)[:4096])
    out = {}
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK, device=device) as dk:
        for name, prec in (("fp32", sd.SD_PREC_MIXED), ("fp64", sd.SD_PREC_FP64)):
            for _ in range(max(1, warmup)):
                dk.pydock_grad(0, poses, prec)
            dt = 0.0
            for _ in range(steps):
                flush.zero_()
                torch.cuda.synchronize(device)
                t0 = time.perf_counter()
                e, g = dk.pydock_grad(0, poses, prec)
                dt += time.perf_counter() - t0
            out[name] = {"poses_per_s": len(poses) * steps / dt, "ms": dt * 1e3 / steps, "grad": g,
                         "h2d_bytes_per_step": int(poses.nbytes + 4 * len(poses)),
                         "d2h_bytes_per_step": int(e.nbytes + g.nbytes)}
        g32, g64 = out["fp32"].pop("grad"), out["fp64"].pop("grad")
        scale = np.maximum(np.abs(g64).max(axis=1, keepdims=True), 1.0)
        out["max_rel_grad_err_fp32_vs_fp64"] = float((np.abs(g32 - g64) / scale).max())
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED, device=device) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, sd.gso_draws(0, S, gso_steps, G))
        dk.step(gso_steps)
        st = dk.get_state(0)
    top = np.argsort(-st.scoring, axis=1)[:, :5]
    sel = np.stack([st.pos[s, top[s]] for s in range(S)]).reshape(-1, cx.pose_len)
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK, device=device) as dk:
        t0 = time.perf_counter()
        _, e0, e1 = dk.refine(0, sel, iters=refine_iters, step=0.5)
        dt = time.perf_counter() - t0
    out["refinement"] = {"poses": int(len(sel)), "iterations": refine_iters, "seconds": dt,
                         "mean_fp64_energy_before": float(e0.mean()), "mean_fp64_energy_after": float(e1.mean()),
                         "fraction_improved": float((e1 < e0).mean()), "max_increase": float((e1 - e0).max())}
    return out


def run_e2e(cfg, steps, device, seed=0):
    """Same metric through the C ABI with host buffers: per step the step's draws go host->device
    from pinned memory and the new state (positions, scores, luciferin) comes back."""
    import torch
    import sparkledock_b200 as sd
    from sparkledock_b200 import _abi
    import ctypes as C
    cxs = make_complexes(cfg)
    tables = sd.synthetic_tables(3)
    dk = sd.Docking(cxs, tables, precision=sd.SD_PREC_MIXED, device=device)
    U = []
    outs = []
    for i, c in enumerate(cxs):
        dk.init_state(i, c.poses)
        u = sd.gso_draws(seed + i, c.n_swarms, steps, c.n_glowworms)
        pin = torch.empty((steps, c.n_swarms, 1, c.n_glowworms), dtype=torch.float64).pin_memory()
        pin.numpy()[:] = np.transpose(u, (1, 0, 2))[:, :, None, :]
        U.append(pin)
        pos = torch.empty((c.n_swarms, c.n_glowworms, c.pose_len), dtype=torch.float64).pin_memory()
        sc = torch.empty((c.n_swarms, c.n_glowworms), dtype=torch.float64).pin_memory()
        lu = torch.empty((c.n_swarms, c.n_glowworms), dtype=torch.float64).pin_memory()
        outs.append((pos, sc, lu))
    L = _abi.lib()
    h2d = sum(c.n_swarms * c.n_glowworms * 8 for c in cxs)
    d2h = sum(c.n_swarms * c.n_glowworms * (c.pose_len + 2) * 8 for c in cxs)
    s0 = dk.stats()
    stream = torch.cuda.ExternalStream(dk.stream, device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t0 = time.perf_counter()
    for t in range(steps):
        for i, c in enumerate(cxs):
            up = U[i][t]
            _abi.check(L.sd_set_draws(dk._ctx, i, C.cast(up.data_ptr(), _abi._dp), 1), "sd_set_draws")
        _abi.check(L.sd_step(dk._ctx, 1, 0), "sd_step")
        for i, c in enumerate(cxs):
            pos, sc, lu = outs[i]
            st = _abi.SwarmState()
            st.pos = C.cast(pos.data_ptr(), _abi._dp)
            st.scoring = C.cast(sc.data_ptr(), _abi._dp)
            st.luciferin = C.cast(lu.data_ptr(), _abi._dp)
            _abi.check(L.sd_get_state(dk._ctx, i, C.byref(st)), "sd_get_state")
    e1.record(stream)
    torch.cuda.synchronize(device)
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    s1 = dk.stats()
    scored = s1["scored_poses"] - s0["scored_poses"]
    dk.close()
    return {"ms": ms, "wall_s": wall, "scored": scored, "h2d": h2d, "d2h": d2h}


SETUP_FILES = ("setup_receptor.pdb", "setup_ligand.pdb")


def setup_structures(cfg, folder):
    """Synthetic compact chains (glycines and alanines, 4.33 atoms per residue) of about the
    first complex's atom counts, written to folder; returns their paths."""
    import sparkledock_b200 as sd
    nr, nl, _ = cfg["complexes"][0]
    paths = [os.path.join(folder, f) for f in SETUP_FILES]
    sd.synthetic_protein_pdb(paths[0], int(round(nr * 3 / 13)), 7)
    sd.synthetic_protein_pdb(paths[1], int(round(nl * 3 / 13)), 8)
    return paths


def time_setup(cfg, folder, device):
    """Wall clock of the setup stages that prepare a docking run from PDB files, on synthetic
    chains of the first complex's size: swarm placement (sd_place_swarms: the receptor-surface
    k-means, sphere filters and starting poses of every swarm x glowworm) and the ANM modes of
    both structures (sd_anm).  Each after one untimed call."""
    import sparkledock_b200 as sd
    rp, lp = setup_structures(cfg, folder)
    flags = sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW
    rec, lig = sd.Structure(rp, flags), sd.Structure(lp, flags)
    S = cfg["complexes"][0][2]
    out = {"receptor_atoms": rec.n_atoms, "ligand_atoms": lig.n_atoms, "swarms": S, "glowworms": G}
    sd.place_swarms(rec, lig, S, G, 10, 10, True, 324324, 324324, device=device)
    t0 = time.perf_counter()
    sd.place_swarms(rec, lig, S, G, 10, 10, True, 324324, 324324, device=device)
    out["placement_ms"] = (time.perf_counter() - t0) * 1e3
    for st, key in ((rec, "anm_receptor_ms"), (lig, "anm_ligand_ms")):
        st.anm(10, 0.5, S, G, device)
        t0 = time.perf_counter()
        st.anm(10, 0.5, S, G, device)
        out[key] = (time.perf_counter() - t0) * 1e3
    return out


def cpu_reference_placement(cfg, folder, device):
    """The reference's own swarm placement (calculate_start_pos, compiled unmodified into
    oracle/_ref/libsdref_anm.so) on the same synthetic chains, wall clock on the host, and whether
    its centres and poses equal sd_place_swarms'."""
    import ctypes as C
    import sparkledock_b200 as sd
    so = os.path.join(ROOT, "oracle", "_ref", "libsdref_anm.so")
    if not os.path.exists(so):
        return {"value": None, "error": "reference harness not built"}
    rp, lp = [os.path.join(folder, f) for f in SETUP_FILES]
    S = cfg["complexes"][0][2]
    dp = C.POINTER(C.c_double)
    L = C.CDLL(so)
    L.ref_start_positions.argtypes = [C.c_char_p, C.c_char_p] + [C.c_int] * 10 + [C.c_double, dp, dp]
    cent = np.zeros((S, 3))
    poses = np.zeros((S, G, 27))
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)  # the reference reports its progress on stdout; keep stdout for the JSON line
    try:
        t0 = time.perf_counter()
        L.ref_start_positions(rp.encode(), lp.encode(), 1, 1, 1, S, G, 324324, 324324, 10, 10, 1, 10.0,
                              cent.ctypes.data_as(dp), poses.ctypes.data_as(dp))
        dt = time.perf_counter() - t0
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    flags = sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW
    c2, p2 = sd.place_swarms(sd.Structure(rp, flags), sd.Structure(lp, flags), S, G, 10, 10, True, 324324, 324324,
                             device=device)
    return {"placement_ms": dt * 1e3, "cores": 1, "kind": "reference",
            "bit_identical": bool(np.array_equal(cent, c2) and np.array_equal(poses, p2))}


def product_library_mapped() -> bool:
    """Whether this process has the product library (libsparkle_b200.so) mapped."""
    try:
        with open("/proc/self/maps") as f:
            return "libsparkle_b200.so" in f.read()
    except OSError:
        return False


def cpu_reference_rate(cfg, budget_s=12.0, seed=0, clean=False):
    """The reference's own CPU scoring path (oracle/_ref: its compiled cdfire_calculate_dfire,
    rotate and GSO helpers, OpenMP over swarms) on a bounded sample of the workload: the first
    min(S, cores) swarms of every complex (one swarm per host thread, as the reference runs them),
    all sampled complexes stepped together from the start until the time budget is spent (at
    least one step).  Each complex's poses and time are scaled by S / sampled swarms, so the rate
    is that of the workload's own mix of complexes.  Falls back to the oracle's C restatement when
    the reference harness was not built.  Inputs come from the oracle's restatement of the
    synthetic generator (bit-identical to the product's), so this leg never loads the product
    library; with clean=True that is checked before timing."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import (OracleState, OracleSynthComplex, OracleSystem, oracle_draws, oracle_step, oracle_tables,
                             ref, ref_available, ref_step)
    cores = os.cpu_count() or 1
    cs = cfg["complexes"]
    kind = "reference" if ref_available() else "port"
    if kind == "reference":
        ref()
    tables = oracle_tables(3)
    samples = [min(S, cores) for _, _, S in cs]
    systems = []
    for i, ((a, b, S), k) in enumerate(zip(cs, samples)):
        cx = OracleSynthComplex(a, b, k, G, 10, 10, seed=100 + i)
        systems.append((OracleSystem(cx, tables, cr_math=0), OracleState(k, G, cx.pose_len, cx.poses),
                        oracle_draws(seed + i, k, 100, G)))
    if clean and product_library_mapped():
        raise RuntimeError("the reference arm has the product library mapped")
    scored = [0] * len(cs)
    secs = [0.0] * len(cs)
    steps = 0
    t0 = time.perf_counter()
    while steps < 100:
        for i, (osys, st, U) in enumerate(systems):
            t1 = time.perf_counter()
            if kind == "reference":
                scored[i] += ref_step(osys, st, U[:, steps, :], cores)
            else:
                before = st.moved.copy(), st.step.copy()
                oracle_step(osys, st, U[:, steps, :], nthreads=cores)
                scored[i] += int(((before[0] == 1) | (before[1] == 0)).sum())
            secs[i] += time.perf_counter() - t1
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    w = [S / k for (_, _, S), k in zip(cs, samples)]
    value = sum(wi * n for wi, n in zip(w, scored)) / sum(wi * t for wi, t in zip(w, secs))
    sample = ", ".join(f"{k}/{S}" for k, (_, _, S) in zip(samples, cs))
    return {"value": value, "unit": "scored poses/s", "cores": cores, "kind": kind,
            "sample": f"swarms {sample} (of each complex) x {G} glowworms, {steps} GSO steps from the start "
                      f"({sum(scored)} poses rescored in {dt:.1f} s wall clock, OpenMP over swarms; each "
                      f"complex's poses and time scaled to its full swarm count)",
            "steps_per_s_sample": steps / dt, "product_library_mapped": product_library_mapped()}


def rank_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def reduce_max_sum(dist, t_ms, scored, device):
    """max of times and sum of scored poses over ranks (identity for one rank)."""
    if dist is None:
        return t_ms, scored
    import torch
    t = torch.tensor([t_ms], dtype=torch.float64, device=device)
    s = torch.tensor([float(scored)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    return float(t.item()), int(s.item())


def measure(cfg, name, args, device, flush, dist, energy_every=0):
    """The workload of one configuration: the timed mixed (or the configuration's precision)
    steps, then the plain FP64 kernels over the same trajectory for the mixed-vs-FP64 ratio."""
    run = run_gpu(cfg, cfg["precision"], args.steps, args.warmup, device, flush, per_step=args.per_step,
                  energy_every=energy_every)
    t_ms, scored = reduce_max_sum(dist, sum(run["ms"]), run["scored"], device)
    _, pairs_all = reduce_max_sum(dist, 0.0, run["pairs"], device)  # every rank takes part
    value = scored / (t_ms / 1e3)
    out = {"run": run, "t_ms": t_ms, "scored": scored, "pairs_all": pairs_all, "value": value}
    extra = {}
    if not args.no_fp64 and cfg["precision"] == "mixed":
        # the FP64 runs take the same trajectory; on the large configurations they are bounded to
        # cmp_steps timed steps (the brute-force FP64 step costs seconds there), and the mixed rate
        # they are compared with is measured again over the same steps
        cmp_steps = min(args.steps, cfg.get("cmp_steps", args.steps))
        ref_value = value
        if cmp_steps < args.steps:
            r = run_gpu(cfg, "mixed", cmp_steps, args.warmup, device, flush)
            tm, sc = reduce_max_sum(dist, sum(r["ms"]), r["scored"], device)
            r["ctx"].close()
            ref_value = sc / (tm / 1e3)
        for pname in ("fp64", "fp64_ref"):
            r = run_gpu(cfg, pname, cmp_steps, args.warmup, device, flush)
            tm, sc = reduce_max_sum(dist, sum(r["ms"]), r["scored"], device)
            r["ctx"].close()
            extra[pname] = {"value": sc / (tm / 1e3), "ms_per_step": tm / cmp_steps,
                            "steps_per_s": cmp_steps / (tm / 1e3), "scored_poses": sc, "timed_steps": cmp_steps,
                            "speedup_mixed": ref_value / (sc / (tm / 1e3))}
            # the same algorithmic work as the mixed line (8 Nr Nl flops per scored pose, or 8 flops
            # per in-cutoff pair at the mixed run's pairs per pose on the large receptor) over the
            # nominal FP64 vector pipe: 148 SMs x 64 lanes x 2 at the measured max SM clock
            fp64_peak = 148 * 64 * 2 * (measured_peaks()[0].get("sm_max_mhz", 1965.0) * 1e6) / 1e12
            per_pose = (8.0 * brute_pairs_per_pose(cfg) if name != "c3" else 8.0 * pairs_all / max(1, scored))
            ach = per_pose * sc / (tm / 1e3) / 1e12
            extra[pname]["roofline"] = {"bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                                        "frac": ach / fp64_peak,
                                        "peak_source": "nominal FP64 vector pipe (148 SMs x 64 lanes x 2) at the "
                                                       "measured max SM clock"}
    out["mixed_vs_fp64"] = extra
    errs = run["energy_err"]
    if errs:
        out["per_step_energy_error"] = {
            "steps_checked": len(errs), "every": energy_every,
            "max_rel_energy_err": max(e["max_rel_energy_err"] for e in errs),
            "max_rel_score_err": max(e["max_rel_score_err"] for e in errs),
            "poses_checked": sum(e["poses"] for e in errs), "tolerance": 1e-5,
            "reference": "plain FP64 kernel (bit-identical to the FP64 oracle) on the poses each step rescored",
            "per_step_max_rel_energy_err": [e["max_rel_energy_err"] for e in errs]}
    return out


def roofline_of(cfg, name, m, args, peaks, peak_src):
    """Roofline of the timed steps: the scorer's work over the FP32 vector pipe (the scorer is
    neither HBM- nor tensor-shaped: its tables stay in L2 and its distance contraction has K = 3).
    Primary: 8 flops per receptor-ligand pair inside the cutoff (the work the culled kernel does,
    counted by the kernel); beside it the brute-force-equivalent 8 Nr Nl flops per scored pose
    (the reference's formulation of the DFIRE sum).  Time: the timed GSO steps (scorer ~99 %)."""
    stats = m["run"]["stats"]
    t_s = m["t_ms"] / 1e3
    mixed = cfg["precision"] == "mixed"
    lanes = 128 if mixed else 64  # FP32 or FP64 vector lanes per SM
    vec_peak = 148 * lanes * 2 * (peaks.get("sm_max_mhz", 1965.0) * 1e6) / 1e12
    cut_tflops = 8.0 * m["pairs_all"] / t_s / 1e12
    brute = 8.0 * brute_pairs_per_pose(cfg) * m["scored"] / t_s / 1e12
    out = {"bound": "fp32" if mixed else "fp64", "achieved": cut_tflops, "peak": vec_peak, "unit": "TFLOP/s",
            "frac": cut_tflops / vec_peak,
            "work": "8 flops per receptor-ligand pair inside the 15 A cutoff (counted by the kernel)",
            "pairs_per_s": m["pairs_all"] / t_s,
            "table_bytes_per_s": 8.0 * m["pairs_all"] / t_s,
            "traffic": DRAM_BYTES_PER_LAUNCH + DRAM_BYTES_PER_SCORED_POSE * m["scored"] / args.steps,
            "traffic_unit": "bytes per launch (DRAM, ncu: fixed + per rescored pose)",
            "peak_source": f"nominal {'FP32' if mixed else 'FP64'} vector pipe (148 SMs x {lanes} lanes x 2) at the "
                           f"measured max SM clock {peaks.get('sm_max_mhz', 1965.0):.0f} MHz "
                           f"({peak_src} peaks file has no FP32 or FP64 vector figure)",
            "hbm_frac": (DRAM_BYTES_PER_LAUNCH * args.steps / t_s +
                         DRAM_BYTES_PER_SCORED_POSE * m["value"]) / 1e9 / peaks.get("hbm_gbs", 6650.0),
            "brute_force_equivalent": {"tflops": brute, "frac": brute / vec_peak,
                                       "work": "8 Nr Nl flops per scored pose"},
            "per_scored_pose": {"pairs_in_cutoff": stats["pairs_in_cutoff"] / max(1, stats["scored_poses"]),
                                "pairs_evaluated": stats["pairs_evaluated"] / max(1, stats["scored_poses"]),
                                "pairs_brute_force": brute_pairs_per_pose(cfg)}}
    if mixed:  # the mixed scorer's measured instructions and L1 wavefronts per in-cutoff pair
        clk = peaks.get("sm_max_mhz", 1965.0) * 1e6
        ceiling = 148 * 4 * clk / WARP_INSTR_PER_PAIR
        out["issue_bound"] = {"warp_instructions_per_pair": WARP_INSTR_PER_PAIR, "ceiling_pairs_per_s": ceiling,
                              "frac": m["pairs_all"] / t_s / ceiling}
        ceiling = 148 * clk / L1_WAVEFRONTS_PER_PAIR
        out["l1_bound"] = {"wavefronts_per_pair": L1_WAVEFRONTS_PER_PAIR, "ceiling_pairs_per_s": ceiling,
                           "frac": m["pairs_all"] / t_s / ceiling}
    return out


def config_of(cfg, args):
    return {"workload": cfg["workload"], "complexes": [list(c) for c in cfg["complexes"]], "glowworms": G,
            "anm_modes": [10, 10], "gso_steps": args.warmup + args.steps, "scoring": "dfire",
            "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{args.gpus}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=97)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison runs")
    ap.add_argument("--no-c1", action="store_true", help="skip the single-complex leg of the batched workload")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--swarms", type=int, default=0, help="override the swarm count (profiling of a smaller case)")
    ap.add_argument("--precision", default="", choices=["", "mixed", "fp64", "fp64_ref"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-setup", action="store_true", help="skip the setup-stage and clustering timings")
    ap.add_argument("--per-step", action="store_true", help="record scored poses and time of every timed step")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.swarms:
        cfg["complexes"] = [(nr, nl, min(s, args.swarms)) for nr, nl, s in cfg["complexes"]]
        cfg["workload"] += f" (swarms capped at {args.swarms})"
    if args.precision and args.precision != cfg.get("precision"):
        cfg["precision"] = args.precision
        cfg["workload"] = cfg["workload"].replace("mixed precision", args.precision + " precision")
    rank, world, local = rank_env()
    config = config_of(cfg, args)

    if args.config == "c4":
        if rank == 0:
            import torch
            torch.cuda.set_device(0)
            flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=0)
            with Clocks(0) as clk:
                res = run_c4(cfg, 0, args.warmup + args.steps, args.steps, args.warmup, flush)
            f32 = res["fp32"]
            print(json.dumps({"metric": "pyDock-style adjoint poses/s (energy + 26-dim gradient, host buffers)",
                              "value": f32["poses_per_s"], "unit": "poses/s", "n_gpus": 1, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": f32["ms"], "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "f32 pairs, f64 sums",
                              "data": "synthetic", "config": config, "gpu_launches": args.steps,
                              "timing": "wall clock around each synchronous call; the API takes host buffers, so "
                                        "value and e2e are the same measurement",
                              "e2e": {"value": f32["poses_per_s"], "unit": "poses/s",
                                      "h2d_bytes_per_step": f32["h2d_bytes_per_step"],
                                      "d2h_bytes_per_step": f32["d2h_bytes_per_step"]},
                              "clocks": clk.summary(), **res}))
        return

    if args.impl == "reference":
        # the reference's own CPU path on rank 0 only; inputs from the oracle, the product library
        # is never loaded in this process (checked before timing)
        if rank != 0:
            return
        cb = cpu_reference_rate(cfg, args.cpu_budget, clean=True)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "scored poses/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cb["value"], "unit": "scored poses/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "product_library_mapped": cb["product_library_mapped"]}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = dist_mod
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    # the configuration's own steps: energies checked every 10th step on the batched workload (its
    # state is 138 MB), every step otherwise; the check runs between steps, outside the events
    energy_every = 0 if cfg["precision"] != "mixed" else (10 if len(cfg["complexes"]) > 1 else 1)
    barrier()
    with Clocks(device) as clk:
        m = measure(cfg, args.config, args, device, flush, dist, energy_every=energy_every)
    barrier()
    run = m["run"]
    stats = run["stats"]
    spot = fp64_spot_check(run["ctx"], run["cxs"]) if cfg["precision"] == "mixed" else None
    clustering = None if args.no_setup else time_clustering(run["ctx"], run["cxs"])
    run["ctx"].close()
    setup_dir = tempfile.mkdtemp(prefix="sd_setup_") if rank == 0 else None
    setup = time_setup(cfg, setup_dir, device) if rank == 0 and not args.no_setup else None

    # the single-complex workload beside the batched one: its own rate and mixed-vs-FP64 ratio
    c1 = None
    if args.config == "c2" and not args.no_c1 and not args.swarms and not args.precision:
        cfg1 = dict(CONFIGS["c1"])
        with Clocks(device) as clk1:
            m1 = measure(cfg1, "c1", args, device, flush, dist, energy_every=1)
        m1["run"]["ctx"].close()
        c1 = {"workload": cfg1["workload"], "complexes": [list(c) for c in cfg1["complexes"]],
              "value": m1["value"], "unit": "scored poses/s", "ms_per_step": m1["t_ms"] / args.steps,
              "steps_per_s": args.steps / (m1["t_ms"] / 1e3), "mixed_vs_fp64": m1["mixed_vs_fp64"],
              "per_step_energy_error": m1.get("per_step_energy_error"), "clocks": clk1.summary(),
              "autotuner": m1["run"]["tuning"]}

    if args.no_e2e:
        e2e = {"ms": float("nan"), "wall_s": None, "scored": 0, "h2d": 0, "d2h": 0}
    else:
        e2e = run_e2e(cfg, args.steps, device)
    et, es = reduce_max_sum(dist, e2e["ms"], e2e["scored"], device)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peaks, peak_src = measured_peaks()
    clocks = clk.summary()
    t_ms = m["t_ms"]
    line = {
        "metric": METRIC, "value": m["value"], "unit": "scored poses/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "steps_per_s": args.steps / (t_ms / 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16/f32 pair tests, f64 table sums and GSO" if cfg["precision"] == "mixed" else "f64",
        "data": "synthetic (seeded globules, N(0,1) DFIRE table)", "config": config,
        "gpu_launches": 2 * args.steps,
        "e2e": {"value": es / (et / 1e3), "unit": "scored poses/s", "h2d_bytes_per_step": e2e["h2d"],
                "d2h_bytes_per_step": e2e["d2h"], "wall_s": e2e["wall_s"]},
        "clocks": clocks,
        "mixed_vs_fp64": m["mixed_vs_fp64"],
        "per_step_energy_error": m.get("per_step_energy_error"),
        "autotuner": run["tuning"],
        "fp64_spot_check": spot,
        "c1": c1,
        "final_clustering": clustering,
        "setup": setup,
        **({"per_step": {"scored_poses": run["per_step"], "pairs_in_cutoff": run["per_step_pairs"], "ms": run["ms"]}}
           if args.per_step else {}),
        "edge_counts": {k: stats[k] for k in ("pairs_fallback", "edge_d2_zero", "edge_d2_cutoff", "edge_u_zero",
                                              "edge_shortfall")},
    }
    if stats.get("pairs_in_cutoff"):
        line["roofline"] = roofline_of(cfg, args.config, m, args, peaks, peak_src)
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = {k: v for k, v in cpu_reference_rate(cfg, args.cpu_budget).items()
                                    if k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        if setup is not None:
            try:
                setup["reference_cpu"] = cpu_reference_placement(cfg, setup_dir, device)
            except Exception as e:
                setup["reference_cpu"] = {"value": None, "error": str(e)[:200]}
    shutil.rmtree(setup_dir, ignore_errors=True)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
