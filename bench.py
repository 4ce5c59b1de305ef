#!/usr/bin/env python
"""Throughput of EDIPIC-2D's per-step particle cycle (push + MCC + deposit, with the FFT_X field solve) on B200.

Workload (default): the 1024x1024-cell periodic-x plasma with 200 electrons and 200 Ar+ per cell
(419,430,400 particles), B = 10 mT at 30 degrees in plane, e-Ar (elastic, excitation, ionisation) and Ar+-Ar
charge exchange, N_subcycles = 1, mixed precision (int32 cell + FP32 offsets/velocities, int64 fixed-point
deposit), tile sort every 20 steps (the configuration's period; the timed window holds whole sort periods, and a
partial one is charged its share of a separately timed sort). Synthetic deck and initial plasma (no dataset is
involved).

One step = one pass of MainProg's cycle (pic2d_MainProgram.f90:151-309): density, FFT_X solve and E, electron
push+deposit+MCC, ion push+deposit+RCX, appends. value = (electrons + ions) * steps / device time of the timed
steps (CUDA events on the library's stream). e2e = the same steps driven through the C ABI in the call order
a Fortran host uses, with the per-step host reads of the collision counters.

--impl reference times the CPU restatement of the reference routines (the oracle: the reference's Fortran
cannot be built in this image) on the host cores, on a bounded sample of the same workload (its physics and
particles per cell on a 256 x 128-cell grid), without loading the device library.
Multi-GPU (torchrun): the ranks share one cluster's particles (each GPU pushes args.ppc electrons and ions per cell
over the whole grid, so the particles per cell grow with N: weak scaling); the int64 fixed-point densities are summed
over the ranks with an NCCL all-reduce after every step and every rank solves the same field. Device time is the max
over ranks.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "edipic-2d_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "particle-steps/s (push+MCC+deposit); Poisson ms/step learned vs plain, 1×B200"
BYTES_PER_PARTICLE_STEP = {"mixed": 52, "fp64": 84}


def workload_desc(args):
    per = " per GPU" if getattr(args, "world", 1) > 1 else ""
    return (f"{args.config}: {args.cells_x}x{args.cells_y} cells, {args.ppc} e- + {args.ppc} Ar+ per cell{per}, "
            f"{'B 10 mT at 30 deg, ' if args.config == 'cfg1' else ''}e-Ar MCC + Ar+-Ar RCX, FFT_X, "
            f"{args.precision} precision, sort every {args.sort_every}")


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu_index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self, min_samples=3):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t0 = time.time()
        while len(self.rows) < min_samples and time.time() - t0 < 3.0:
            time.sleep(0.05)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for k, n in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _decks_module():
    """The synthetic-deck writer (edipic_b200/decks.py, which writes plain text files), loaded from its file so that
    the CPU legs import nothing else of the device package and never load libedipic_b200.so."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "edipic_decks", os.path.join(ROOT, "edipic-2d_b200", "edipic_b200", "decks.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _oracle_cycle_rate(config, ncx, ncy, ppc, threads, seconds, seed=1):
    """particle-steps/s of the oracle's cycle (FP64; OpenMP on `threads` threads) on a deck of the given
    configuration and grid, with the plasma of its init_particles.dat (uniform positions, Maxwellian electrons at
    init_Te and ions at init_Ti, DISTRIBUTE_PARTICLES), stepped for about `seconds` after one untimed step. The deck
    is read by the oracle's own reader."""
    import numpy as np

    import pyoracle
    decks = _decks_module()
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.write_deck(tmp, config, ncx=ncx, ncy=ncy, ppc=ppc)
        dk = pyoracle.read_deck(d)
        rng = np.random.default_rng(seed)
        n = ncx * ncy * ppc
        x = rng.uniform(0, ncx, n)
        y = rng.uniform(0, ncy, n)
        # factor_convert = sqrt(T / T_scale) / N_max_vel per component of exp(-u^2) (pic2d_CurProblemValues.f90:3127)
        fe = np.sqrt(dk["init_Te_eV"] / dk["T_e_eV"]) / dk["N_max_vel"]
        fi = np.sqrt(dk["ions"][0]["init_Ti_eV"] / (dk["T_e_eV"] * dk["ions"][0]["Ms"])) / dk["N_max_vel"]
        ve = rng.normal(0, fe / np.sqrt(2.0), (3, n))
        vi = rng.normal(0, fi / np.sqrt(2.0), (3, n))
        oc = pyoracle.OracleCycle(d, (x, y, ve[0], ve[1], ve[2]), (x, y, vi[0], vi[1], vi[2]), seed=seed,
                                  nthreads=threads)
        oc.step(1)
        done, steps, t0 = 0, 0, time.perf_counter()
        while True:
            done += oc.step(1)
            steps += 1
            el = time.perf_counter() - t0
            if el > seconds or steps >= 5000:
                break
    return done / el, steps, el, 2 * n


def host_cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(args, seconds=12.0):
    """The oracle's cycle (the FP64 restatement of the reference routines) on the host cores: the line's
    workload per particle (its configuration's physics and particles per cell, the grid sampled to 256 x 128 cells)
    on all host threads and on one thread, plus the reference's own CPU-runnable case (cfg0: 128 x 128 cells,
    64 + 64 per cell, FFT_X) on all threads and on one thread. Each leg steps for about `seconds`."""
    threads = os.cpu_count() or 1
    sx, sy = min(args.cells_x, 256), min(args.cells_y, 128)
    v_all, st_all, el_all, n_all = _oracle_cycle_rate(args.config, sx, sy, args.ppc, threads, seconds)
    v_one, st_one, el_one, _ = _oracle_cycle_rate(args.config, sx, sy, args.ppc, 1, seconds)
    v_c0, st_c0, el_c0, n_c0 = _oracle_cycle_rate("cfg0", 128, 128, 64, threads, seconds)
    v_c01, st_c01, el_c01, _ = _oracle_cycle_rate("cfg0", 128, 128, 64, 1, seconds)
    return {"value": v_all, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "cpu_model": host_cpu_model(),
            "sample": f"{args.config} physics on {sx}x{sy} cells x {args.ppc}+{args.ppc} per cell ({n_all} "
                      f"particles), {st_all} steps in {el_all:.1f} s on {threads} threads; FP64 oracle cycle incl. "
                      f"FFT_X (the reference's Fortran/MPI/PETSc cannot be built in this image)",
            "one_thread": {"value": v_one, "steps": st_one, "seconds": el_one},
            "cfg0_all_threads": {"value": v_c0, "steps": st_c0, "seconds": el_c0,
                                 "sample": f"cfg0: 128x128 cells x 64+64 per cell ({n_c0} particles), FFT_X"},
            "cfg0_one_thread": {"value": v_c01, "steps": st_c01, "seconds": el_c01}}


def line_config(args, world=1, per_gpu_particles=None):
    """The `config` object of the JSON line, the same for both arms."""
    c = {"workload": workload_desc(args), "cells": [args.cells_x, args.cells_y],
         "particles_per_gpu": int(per_gpu_particles if per_gpu_particles is not None
                                  else 2 * args.cells_x * args.cells_y * args.ppc),
         "parallelism": (f"one cluster over {world} GPUs: particles split, densities summed by NCCL all-reduce, "
                         "field replicated" if world > 1 else "1 GPU"),
         "l2": "particle arrays (>10 GB) exceed L2 each step",
         "sort": f"tile sort every {args.sort_every} steps, amortised in ms_per_step"}
    return c


def fp64_cycle_leg(args, stream_of):
    """The same workload through the plain FP64 device path (84 B per particle-step, no sort): the comparison the
    mixed-precision cycle is quoted against."""
    from edipic_b200 import PREC_FP64, Simulation, decks
    import torch
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.write_deck(tmp, args.config, ncx=args.cells_x, ncy=args.cells_y, ppc=args.ppc)
        with Simulation(d, precision=PREC_FP64, sort_every=0, fuse_collisions=True, seed=1000) as sim:
            sim.distribute_particles(args.ppc)
            stream = stream_of(sim)
            for _ in range(3):
                sim.step(1)
            c0 = sim.counters()
            steps = 10
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            sim.step(steps)
            b.record(stream)
            b.synchronize()
            t = a.elapsed_time(b) / 1e3
            c1 = sim.counters()
    n = 0.5 * (c0.n_particles[0] + c0.n_particles[1] + c1.n_particles[0] + c1.n_particles[1])
    return {"value": n * steps / t, "unit": "particle-steps/s", "ms_per_step": 1e3 * t / steps, "steps": steps,
            "path": "FP64 particles and FP64 atomic deposit, same kernels' FP64 variants, whole cycle incl. FFT_X"}


def network_leg():
    """The learned warm start's convolutions on the tensor cores: each of the 14 layers of the encoder-decoder timed
    alone at the inference shape (one image of the 513 x 513-node grid padded to 576 x 576) and at the training shape
    (4 images), and the whole forward pass. FLOPs = 2 x pixels x 9 x c_in x c_out per layer. A layer's device time
    (`us`, the FLOP rate) is 20 calls replayed from a CUDA graph; `call_us` is the same calls made one by one from
    Python, with the host's call and launch overhead."""
    # (the image is the 513 x 513-node grid padded to a multiple of 64)
    import torch
    from edipic_b200 import library, warmstart
    lib = library()
    H = W = warmstart.padded(513)   # the 513 x 513-node grid of the inner-object geometry
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
        peak_kind = "measured"
    except Exception:
        peak, peak_kind = 1590.0, "fallback"
    p = warmstart.POOL
    scale = [1, 1, p, p, p ** 2, p ** 2, p ** 3, p ** 3, p ** 2, p ** 2, p, p, 1, 1]
    net = warmstart.WarmStartNet(seed=0)
    out = {"shape": f"{H}x{W}", "peak_tflops": peak, "peak_kind": peak_kind}
    st = torch.cuda.Stream()
    for nb in (1, 4):
        tot_t, tot_f, tot_c, per = 0.0, 0.0, 0.0, []
        for l, (ci, co) in enumerate(warmstart.LAYERS):
            h, w = H // scale[l], W // scale[l]
            x = torch.randn(nb, h, w, ci, device="cuda").to(torch.bfloat16)
            y = torch.empty(nb, h, w, co, device="cuda", dtype=torch.bfloat16)
            wo, bo, _, _ = net.convs[l]
            wb, bb = net.theta_bf[wo:bo], net.theta[bo:bo + co].detach()
            args = (nb, h, w, C.c_void_p(x.data_ptr()), ci, None, 0, C.c_void_p(wb.data_ptr()),
                    C.c_void_p(bb.data_ptr()), co, 1, C.c_void_p(y.data_ptr()), C.c_void_p(st.cuda_stream))
            torch.cuda.synchronize()
            for _ in range(3):
                lib.edp_nn_conv3x3_fwd(*args)
            reps = 20
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            # per call, with the host's call overhead (ctypes, launch)
            e0.record(st)
            for _ in range(reps):
                lib.edp_nn_conv3x3_fwd(*args)
            e1.record(st)
            e1.synchronize()
            t_call = e0.elapsed_time(e1) / 1e3 / reps
            # device time: the same calls replayed from a CUDA graph captured on the same stream
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=st):
                for _ in range(reps):
                    lib.edp_nn_conv3x3_fwd(*args)
            g.replay()
            torch.cuda.synchronize()
            e0.record(st)
            with torch.cuda.stream(st):
                g.replay()
            e1.record(st)
            e1.synchronize()
            t = e0.elapsed_time(e1) / 1e3 / reps
            del g
            f = 2.0 * nb * h * w * 9 * ci * co
            tot_t += t
            tot_c += t_call
            tot_f += f
            per.append({"layer": l, "cin": ci, "cout": co, "hw": [h, w], "us": 1e6 * t, "call_us": 1e6 * t_call,
                        "tflops": f / t / 1e12})
        x = torch.randn(nb, H, W, 32, device="cuda").to(torch.bfloat16)
        cs = torch.cuda.current_stream()   # the training wrappers launch on torch's current stream
        with torch.no_grad():
            for _ in range(3):
                net.forward(x)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cs)
            for _ in range(10):
                net.forward(x)
            e1.record(cs)
            e1.synchronize()
        fwd = e0.elapsed_time(e1) / 10
        out[f"batch{nb}"] = {"conv_ms": 1e3 * tot_t, "conv_gflop": tot_f / 1e9, "conv_tflops": tot_f / tot_t / 1e12,
                             "frac": tot_f / tot_t / 1e12 / peak, "conv_ms_per_call": 1e3 * tot_c,
                             "forward_ms": fwd, "layers": per}
    return out


def poisson_leg(args, stream_of, warmup=10, steps=30, only=None):
    """Poisson ms/step on the inner-object geometry (512 x 512 cells, metal walls at 0 V, a 64 x 32-cell metal
    rectangle at -100 V centred at (256, 128), 100 e- + 100 Ar+ per cell, the full collision set): each step of the
    cycle solves with CG to a 1e-8 relative residual from the previous step's potential. Timed by CUDA events
    around each solve (density, CG with its convergence reads, E)."""
    from edipic_b200 import PRECOND_MG, PRECOND_NONE, WARM_LEARNED, WARM_PREVIOUS, Simulation, decks, warmstart
    import torch
    out = {"workload": "cfg2: 512x512 cells, inner metal rectangle 64x32 cells at -100 V, 100+100 per cell, "
                       "CG to 1e-8 relative residual, previous-step (plain) or learned warm start", "rtol": 1e-8}
    theta = None
    wpath = os.path.join(ROOT, "edipic-2d_b200", "weights", "warmstart_cfg3.npz")
    if os.path.exists(wpath):
        try:
            theta = warmstart.load_blob(wpath)
            out["weights"] = os.path.relpath(wpath, ROOT)
        except ValueError as e:   # parameters of another network layout
            out["learned"] = {"unavailable": str(e)}
    runs = [("plain_mg", PRECOND_MG, WARM_PREVIOUS), ("plain_nopc", PRECOND_NONE, WARM_PREVIOUS)]
    if theta is not None:
        runs += [("learned_mg", PRECOND_MG, WARM_LEARNED), ("learned_nopc", PRECOND_NONE, WARM_LEARNED)]
    elif "learned" not in out:
        out["learned"] = {"unavailable": "no trained weights (edipic_b200.train_warmstart writes them)"}
    if only:
        runs = [r for r in runs if r[0] in only]
    for name, pc, warm in runs:
        with tempfile.TemporaryDirectory() as tmp:
            d = decks.write_deck(tmp, "cfg2")
            with Simulation(d, sort_every=80, fuse_collisions=True, seed=2000) as sim:
                sim.set_cg_preconditioner(pc)
                if theta is not None:
                    sim.load_warm_start(theta)
                sim.distribute_particles(100)
                stream = stream_of(sim)
                lib, ctx, chk = sim.lib, sim.ctx, sim._check
                it = C.c_int32()
                times, iters = [], []
                for k in range(warmup + steps):
                    chk(lib.edp_update_wall_potentials(ctx, k), "wall")
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    chk(lib.edp_field_cg(ctx, 1e-8, 200000, warm if k > 0 else WARM_PREVIOUS, C.byref(it)), "cg")
                    b.record(stream)
                    chk(lib.edp_advance_electrons(ctx), "adv_e")
                    chk(lib.edp_advance_ions(ctx), "adv_i")
                    chk(lib.edp_collide_en(ctx, None), "en")
                    chk(lib.edp_collide_rcx(ctx, None), "rcx")
                    chk(lib.edp_end_ion_cycle(ctx), "end")
                    if k >= warmup:
                        b.synchronize()
                        times.append(a.elapsed_time(b))
                        iters.append(it.value)
        out[name] = {"ms_per_step": sum(times) / len(times), "cg_iterations_mean": sum(iters) / len(iters),
                     "cg_iterations_max": max(iters), "steps": steps,
                     "preconditioner": "multigrid V(2,2) RB-GS" if pc == PRECOND_MG else "none (Jacobi = plain)",
                     "warm_start": "learned" if warm == WARM_LEARNED else "previous step"}
    for pcn in ("mg", "nopc"):
        if f"learned_{pcn}" in out:
            pl, le = out[f"plain_{pcn}"], out[f"learned_{pcn}"]
            out[f"learned_over_plain_{pcn}"] = {
                "cg_iteration_ratio": pl["cg_iterations_mean"] / max(le["cg_iterations_mean"], 1e-9),
                "ms_ratio": pl["ms_per_step"] / le["ms_per_step"]}
    return out


def warm_start_ceiling(args, stream_of, warmup=12, samples=3):
    """How close a warm start must be to cut CG work: on the cfg2 geometry (512 x 512 cells, metal rectangle at
    -100 V, 100 + 100 per cell) after `warmup` steps of the cycle, for `samples` later steps, the converged potential
    phi* (relative residual 1e-13) and the previous one give starts phi_prev + (1 - eps) (phi* - phi_prev) of known
    accuracy eps; CG iterations to 1e-8 from each, plain and multigrid-preconditioned. eps = 1 is the plain previous
    start. With trained weights, the network's guess is placed on the same scale (its eps = |guess - phi*| /
    |phi* - phi_prev| in the RMS over the nodes)."""
    import numpy as np

    from edipic_b200 import FIELD_PHI, PRECOND_MG, PRECOND_NONE, WARM_PREVIOUS, WARM_USER, Simulation, decks, warmstart
    eps_list = [1.0, 0.3, 0.1, 0.03, 0.01, 3e-3, 1e-3, 3e-4, 1e-4]
    out = {"workload": "cfg2 geometry, starts phi_prev + (1 - eps)(phi* - phi_prev), CG to 1e-8", "eps": eps_list}
    theta = None
    wpath = os.path.join(ROOT, "edipic-2d_b200", "weights", "warmstart_cfg3.npz")
    if os.path.exists(wpath):
        try:
            theta = warmstart.load_blob(wpath)
        except ValueError:
            theta = None
    iters = {"plain": [[] for _ in eps_list], "mg": [[] for _ in eps_list]}
    net_eps = []
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.write_deck(tmp, "cfg2")
        with Simulation(d, sort_every=20, fuse_collisions=True, seed=2100) as sim:
            if theta is not None:
                sim.load_warm_start(theta)
            sim.distribute_particles(100)
            for k in range(warmup + samples):
                sim.update_wall_potentials(k)
                if k >= warmup:
                    phi_prev = sim.field(FIELD_PHI)
                    guess = sim.predict_warm_start()[0] if theta is not None else None
                    sim.set_cg_preconditioner(PRECOND_MG)
                    sim.solve_potential_with_cg(rtol=1e-13, max_it=200000, warm_start=WARM_PREVIOUS)
                    phi_star = sim.field(FIELD_PHI)
                    dphi = phi_star - phi_prev
                    if guess is not None:
                        net_eps.append(float(np.sqrt(np.mean((guess - phi_star) ** 2) / np.mean(dphi ** 2))))
                    for name, pc in (("plain", PRECOND_NONE), ("mg", PRECOND_MG)):
                        sim.set_cg_preconditioner(pc)
                        for q, eps in enumerate(eps_list):
                            sim.set_field(FIELD_PHI, phi_prev + (1.0 - eps) * dphi)
                            iters[name][q].append(sim.solve_potential_with_cg(rtol=1e-8, max_it=200000,
                                                                              warm_start=WARM_USER))
                    sim.set_cg_preconditioner(PRECOND_MG)
                    sim.set_field(FIELD_PHI, phi_star)
                else:
                    sim.solve_potential_with_cg(rtol=1e-8, max_it=200000, warm_start=WARM_PREVIOUS)
                sim.advance_electrons()
                sim.advance_ions()
                sim.perform_electron_neutral_collisions()
                sim.perform_resonant_charge_exchange()
                sim.end_ion_cycle()
    for name in ("plain", "mg"):
        mean = [float(np.mean(v)) for v in iters[name]]
        out[name] = {"cg_iterations": mean, "ratio_to_previous_start": [mean[0] / max(m, 1e-9) for m in mean]}
    if net_eps:
        out["network_eps"] = float(np.mean(net_eps))
    return out


def run_reference(args):
    """The reference arm: the reference's routines for the path on the host CPU. The reference's Fortran cannot be
    built in this image, so its CPU restatement (the oracle) runs, on all host threads, on the line's workload per
    particle (the grid sampled: cpu_baseline). Only rank 0 works; nothing of the device library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_baseline(args, seconds=20.0)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": cb["unit"], "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": line_config(args),
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    args.world = world
    from edipic_b200 import ELECTRONS, IONS, PREC_FP64, PREC_MIXED, Simulation, cluster, decks
    tmp = tempfile.mkdtemp(prefix=f"edp_bench_{rank}_")
    # the deck's particles per cell (the density normalisation) count all ranks' particles
    d = decks.write_deck(tmp, args.config, ncx=args.cells_x, ncy=args.cells_y, ppc=args.ppc * world)
    prec = PREC_MIXED if args.precision == "mixed" else PREC_FP64
    sim = Simulation(d, precision=prec, sort_every=args.sort_every, fuse_collisions=True, seed=1000)
    lib, ctx = sim.lib, sim.ctx
    if args.push_kernel is not None:
        sim._check(lib.edp_set_push_kernel(ctx, args.push_kernel), "edp_set_push_kernel")
    if args.sort_pass:
        sim._check(lib.edp_set_sort_in_push(ctx, 0), "edp_set_sort_in_push")
    share = cluster.ClusterShare(sim, rank, world)   # disjoint ids; density sums over the ranks
    sim.distribute_particles(args.ppc)
    share.reduce()
    sptr = C.c_void_p()
    lib.edp_get_stream(ctx, C.byref(sptr))
    stream = torch.cuda.ExternalStream(sptr.value)
    chk = sim._check

    def step_plain(ev=None):
        t = sim.counters_cache_t if hasattr(sim, "counters_cache_t") else 0
        chk(lib.edp_update_wall_potentials(ctx, t), "wall")
        if ev:
            ev[0].record(stream)
        chk(lib.edp_field_fftx(ctx, None), "fftx")
        if ev:
            ev[1].record(stream)
        chk(lib.edp_advance_electrons(ctx), "adv_e")
        if ev:
            ev[3].record(stream)
        chk(lib.edp_advance_ions(ctx), "adv_i")
        if ev:
            ev[2].record(stream)
        chk(lib.edp_collide_en(ctx, None), "en")
        chk(lib.edp_collide_rcx(ctx, None), "rcx")
        chk(lib.edp_end_ion_cycle(ctx), "end")
        share.reduce()
        sim.counters_cache_t = t + 1

    for _ in range(args.warmup):
        step_plain()
    # the timed window starts one step after a sort, so that it holds steps // sort_every sorts (a due sort runs in the
    # next step's push, or at the end of the step with --sort-pass); a window that is not a whole number of sort
    # periods is charged the rest of the period's sort by the separately timed sort below
    sort_s = 0.0
    if args.sort_every > 0 and prec == PREC_MIXED:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ts0 = time.perf_counter()
        chk(lib.edp_sort_particles(ctx), "sort")
        torch.cuda.synchronize()
        sort_s = time.perf_counter() - ts0
        if dist:
            tt = torch.tensor([sort_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            sort_s = tt.item()
        step_plain()
    c0 = sim.counters()
    n0 = c0.n_particles[0] + c0.n_particles[1]
    launches0 = c0.kernel_launches
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local if world > 1 else 0)
    clocks.start()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        step_plain(evs[k])
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    c1 = sim.counters()
    n1 = c1.n_particles[0] + c1.n_particles[1]
    launches = c1.kernel_launches - launches0
    t_total = start.elapsed_time(end) / 1e3
    t_field = sum(e[0].elapsed_time(e[1]) for e in evs) / 1e3
    t_push = sum(e[1].elapsed_time(e[2]) for e in evs) / 1e3
    # the push launches of each step (electrons, then ions, with their fused collision epilogues): the steps whose
    # push also wrote the sorted order (the sort steps, by far the longest) are kept apart from the plain ones
    step_push = sorted(e[1].elapsed_time(e[2]) / 1e3 for e in evs)
    n_sort_steps = 0
    if args.sort_every > 0 and prec == PREC_MIXED and not args.sort_pass:
        n_sort_steps = min(args.steps // args.sort_every, len(step_push) - 1)
    plain_push = step_push[:len(step_push) - n_sort_steps]
    t_plain_push = sum(plain_push) / len(plain_push)
    t_sort_push = sum(step_push[len(plain_push):]) / n_sort_steps if n_sort_steps else 0.0
    plain_ev = sorted(evs, key=lambda e: e[1].elapsed_time(e[2]))[:len(plain_push)]
    t_push_e = sum(e[1].elapsed_time(e[3]) for e in plain_ev) / len(plain_ev) / 1e3
    t_push_i = sum(e[3].elapsed_time(e[2]) for e in plain_ev) / len(plain_ev) / 1e3
    if dist:
        tt = torch.tensor([t_total, t_field, t_push, t_plain_push, t_sort_push], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total, t_field, t_push, t_plain_push, t_sort_push = tt.tolist()
        cnt = torch.tensor([float(n0 + n1)], device="cuda", dtype=torch.float64)
        dist.all_reduce(cnt)
        nsum = cnt.item()
    else:
        nsum = float(n0 + n1)
    particle_steps = 0.5 * nsum * args.steps
    sorts_in_window = 0
    if args.sort_every > 0 and prec == PREC_MIXED:
        sorts_in_window = (args.steps + (1 if args.sort_pass else 0)) // args.sort_every
    sort_charge = max(0.0, args.steps / args.sort_every - sorts_in_window) * sort_s if args.sort_every > 0 else 0.0
    t_total += sort_charge
    value = particle_steps / t_total

    # end to end: the drop-in call order of a Fortran host (pic2d_MainProgram.f90:151-309) with its per-step reads
    e2e_steps = args.steps
    cnt_buf = (C.c_int64 * 8)()
    rcx_buf = C.c_int64()
    rho_host = None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    es.record(stream)
    for _ in range(e2e_steps):
        t = sim.counters_cache_t
        chk(lib.edp_gather_charge_density(ctx, IONS, rho_host), "gi")
        chk(lib.edp_gather_charge_density(ctx, ELECTRONS, rho_host), "ge")
        chk(lib.edp_update_wall_potentials(ctx, t), "wall")
        chk(lib.edp_field_fftx(ctx, None), "fftx")
        chk(lib.edp_advance_electrons(ctx), "adv_e")
        chk(lib.edp_advance_ions(ctx), "adv_i")
        chk(lib.edp_collide_en(ctx, cnt_buf), "en")
        chk(lib.edp_collide_rcx(ctx, C.byref(rcx_buf)), "rcx")
        chk(lib.edp_end_ion_cycle(ctx), "end")
        share.reduce()
        sim.counters_cache_t = t + 1
    ee.record(stream)
    ee.synchronize()
    t_e2e = es.elapsed_time(ee) / 1e3
    c2 = sim.counters()
    n2 = c2.n_particles[0] + c2.n_particles[1]
    if dist:
        tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = tt.item()
        cnt = torch.tensor([float(n1 + n2)], device="cuda", dtype=torch.float64)
        dist.all_reduce(cnt)
        ne2e = cnt.item()
    else:
        ne2e = float(n1 + n2)
    e2e = 0.5 * ne2e * e2e_steps / t_e2e

    if rank == 0:
        peak, peak_kind = measured_peaks()
        bpp = BYTES_PER_PARTICLE_STEP[args.precision]
        per_gpu_particles = 0.5 * (n0 + n1)
        achieved = per_gpu_particles * bpp / t_plain_push / 1e9
        traffic = None
        try:
            with open(os.path.join(ROOT, "profiles", "push_traffic.json")) as f:
                tr = json.load(f)
            traffic = tr["dram_bytes_per_particle"][args.precision] * per_gpu_particles
        except Exception:
            pass
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 particles / i64 fixed-point density / f64 field" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": line_config(args, world, per_gpu_particles),
            "sort": {"every": args.sort_every, "sorts_in_window": sorts_in_window, "sort_ms": 1e3 * sort_s,
                     "charged_ms": 1e3 * sort_charge,
                     "where": "separate pass" if args.sort_pass else "in the next push (sorted slots written directly)",
                     "how": "window starts one step after a sort and holds whole sort periods; the rest of a partial "
                            "period is charged from a separately timed sort pass"},
            "poisson_ms_per_step": 1e3 * t_field / args.steps,
            "push_ms_per_step": 1e3 * t_push / args.steps,
            "push": {"plain_step_ms": 1e3 * t_plain_push, "electrons_ms": 1e3 * t_push_e, "ions_ms": 1e3 * t_push_i,
                     "sort_step_ms": 1e3 * t_sort_push, "sort_steps": n_sort_steps},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "basis": f"{bpp} B/particle-step algorithmic / CUDA-event time of the electron and ion "
                                  f"push launches (push + deposit + collision epilogue) of the steps without a sort; "
                                  f"the sort steps, whose push also writes the sorted order, are in push.sort_step_ms; "
                                  f"peak {peak_kind}"},
            "clocks": clk, "gpu_launches": int(launches),
            "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * 8 + 8,
                    "path": "C ABI call sequence of the Fortran host with per-step counter reads"},
        }
    sim.close()
    if rank == 0:
        def stream_of(s):
            ptr = C.c_void_p()
            s.lib.edp_get_stream(s.ctx, C.byref(ptr))
            return torch.cuda.ExternalStream(ptr.value)
        if not args.no_extra_legs and world == 1:
            line["fp64_gpu_cycle"] = fp64_cycle_leg(args, stream_of)
            line["fp64_gpu_cycle"]["mixed_over_fp64"] = value / line["fp64_gpu_cycle"]["value"]
            line["poisson"] = poisson_leg(args, stream_of)
            line["warm_start_ceiling"] = warm_start_ceiling(args, stream_of)
            line["network"] = network_leg()
            line["roofline_conv"] = {"bound": "tensor", "achieved": line["network"]["batch4"]["conv_tflops"],
                                     "peak": line["network"]["peak_tflops"], "unit": "TFLOP/s",
                                     "frac": line["network"]["batch4"]["frac"], "traffic": None,
                                     "basis": "14 tcgen05 convolutions of the warm-start network, 4 x 576 x 576, "
                                              "2 x pixels x 9 x c_in x c_out FLOPs, peak bf16 "
                                              + line["network"]["peak_kind"]}
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="cfg1")
    ap.add_argument("--cells", type=int, nargs=2, default=None, metavar=("NX", "NY"))
    ap.add_argument("--ppc", type=int, default=None)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--sort-every", type=int, default=None,
                    help="tile sort period in steps (default: the configuration's, 20 for cfg1)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-legs", action="store_true", help="skip the FP64-cycle and Poisson legs")
    ap.add_argument("--poisson-only", nargs="*", default=None, metavar="RUN",
                    help="only the Poisson leg (cfg2 geometry), optionally only the named runs "
                         "(plain_mg, plain_nopc, learned_mg, learned_nopc)")
    ap.add_argument("--poisson-steps", type=int, default=30)
    ap.add_argument("--warm-ceiling", action="store_true", help="only the warm-start accuracy leg (cfg2 geometry)")
    ap.add_argument("--sort-pass", action="store_true",
                    help="periodic sorts as a separate pass instead of inside the next push")
    ap.add_argument("--push-kernel", type=int, default=None, choices=[0, 1, 2, 3, 4],
                    help="mixed push over the sorted chunks (edp_set_push_kernel): 0 per-chunk CTAs, 1 streaming "
                         "(bulk copies, 4 particles per thread), 2 streaming (2 per thread, 3 stages), 3 per-chunk "
                         "CTAs with 2 particles per thread, 4 per-chunk CTAs with each thread's next group copied "
                         "ahead by cp.async")
    args = ap.parse_args()
    cfg = _decks_module().CONFIGS[args.config]
    args.cells_x, args.cells_y = args.cells if args.cells else (cfg["ncx"], cfg["ncy"])
    args.ppc = args.ppc or cfg["ppc"]
    if args.sort_every is None:
        args.sort_every = cfg.get("sort_every", 20)
    if args.warmup < 3:
        args.warmup = 3
    if args.poisson_only is not None:
        import torch

        def stream_of(s):
            ptr = C.c_void_p()
            s.lib.edp_get_stream(s.ctx, C.byref(ptr))
            return torch.cuda.ExternalStream(ptr.value)
        print(json.dumps({"poisson": poisson_leg(args, stream_of, warmup=max(args.warmup, 3), steps=args.poisson_steps,
                                                 only=args.poisson_only or None)}))
    elif args.warm_ceiling:
        print(json.dumps({"warm_start_ceiling": warm_start_ceiling(args, None)}))
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
