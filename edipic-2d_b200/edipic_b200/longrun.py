"""Long-run statistical comparison of the mixed-precision device cycle with the plain FP64 device cycle on the
RF-driven periodic configuration (the cfg4 physics: top electrode at 200 V and 13.56 MHz, bottom grounded, e-Ar MCC,
Ar+-Ar charge exchange, ion-induced electron emission of yield 0.1 at both walls), over several seeds. Each run
samples, after a burn-in, the electron energy distribution (EEDF), the electron and ion density profiles across the
gap (COLLECT_*_MOMENTS averaged along x), the electron f(v_x) of CALCULATE_ELECTRON_VDF and the ion flux to each wall.
Two analyses of the per-seed samples: `compare_paired` for runs of the two precisions started from the same seed
(the same initial plasma and random streams): the per-seed differences, their mean over seeds divided by its standard
error, and the smallest bias the test could detect (3 standard errors, relative to the quantity); `compare` (Welch)
for independent seeds.

    python -m edipic_b200.longrun --seeds 8 --steps 12000 --cells 2048 512 --ppc 100 --out longrun.json
"""
import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import ELECTRONS, IONS, PREC_FP64, PREC_MIXED, Simulation, decks

EEDF_EDGES_EV = np.concatenate([[0.0], np.geomspace(0.05, 100.0, 40)])


def run(precision, seed, steps, cells=(64, 64), ppc=64, burn_in=None, sample_every=20, workdir=None):
    """One run of `steps` steps; returns the time-averaged samples of the second half (or after burn_in)."""
    burn_in = steps // 2 if burn_in is None else burn_in
    tmp = tempfile.mkdtemp(dir=workdir)
    d = decks.write_deck(os.path.join(tmp, "deck"), "cfg4", ncx=cells[0], ncy=cells[1], ppc=ppc, steps=steps)
    with Simulation(d, precision=precision, sort_every=20 if precision == PREC_MIXED else 0, seed=seed) as sim:
        sim.distribute_particles(ppc)
        eedf = np.zeros(len(EEDF_EDGES_EV) - 1)
        ne = np.zeros(sim.ny_ref)
        ni = np.zeros(sim.ny_ref)
        fvx = None
        n_samples = 0
        hits0 = None
        for t in range(steps):
            sim.step(1)
            if t + 1 == burn_in:
                c = sim.counters()
                hits0 = np.array(c.ion_hits[:2], dtype=np.float64)
            if t + 1 > burn_in and (t + 1 - burn_in) % sample_every == 0:
                # the EEDF on the device (edp_energy_histogram), normalised by all electrons
                h = sim.energy_histogram(ELECTRONS, EEDF_EDGES_EV).astype(np.float64)
                n_e = max(int(sim.counters().n_particles[0]), 1)
                eedf += h / n_e
                ne += sim.collect_moments(ELECTRONS)[0].mean(axis=1)
                ni += sim.collect_moments(IONS)[0].mean(axis=1)
                v1, _, _ = sim.calculate_vdf(ELECTRONS, (1, 1), 4, 10)
                f = v1[0, 0].astype(np.float64)
                fvx = f / f.sum() if fvx is None else fvx + f / f.sum()
                n_samples += 1
        c = sim.counters()
        flux = (np.array(c.ion_hits[:2], dtype=np.float64) - hits0) / (steps - burn_in)
    return dict(eedf=(eedf / n_samples).tolist(), ne=(ne / n_samples).tolist(), ni=(ni / n_samples).tolist(),
                fvx=(fvx / n_samples).tolist(), ion_flux=flux.tolist(), samples=n_samples)


def zscores(a, b, floor=0.0):
    """|mean_a - mean_b| / sqrt(se_a^2 + se_b^2) per component for per-seed samples a, b [seeds, n]; components
    whose means are both below floor are dropped."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    ma, mb = a.mean(0), b.mean(0)
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    keep = (np.maximum(ma, mb) > floor) & (se > 0)
    return (ma - mb)[keep] / se[keep]


QUANTITIES = (("eedf", 1e-3), ("ne", 0.0), ("ni", 0.0), ("fvx", 1e-3), ("ion_flux", 0.0))


def compare(mixed, fp64):
    """Welch z-scores of every quantity between the two lists of run() results (independent seeds)."""
    out = {}
    for k, floor in QUANTITIES:
        z = zscores([r[k] for r in mixed], [r[k] for r in fp64], floor)
        out[k] = dict(n=int(z.size), max_abs_z=float(np.abs(z).max()) if z.size else 0.0,
                      mean_z2=float((z ** 2).mean()) if z.size else 0.0)
    return out


def compare_paired(mixed, fp64, rel_tol=0.01):
    """Paired analysis of runs with the same seeds (mixed[s] and fp64[s] from the same initial plasma): per component
    the per-seed differences d_s, z = mean(d) / (sd(d) / sqrt(seeds)); and the bias the test could detect, 3 sd(d) /
    sqrt(seeds) relative to the component's mean, as its median over the components (the largest, the smallest).
    Because the pairing removes the seed's own noise, z sees relative biases of 1e-4 and below, which are no physics
    difference; the equivalence score excess_z = max(0, |mean(d)| - rel_tol |m|) / se is the distance, in standard
    errors, by which a component's bias exceeds the tolerance rel_tol of its mean m (0 while it stays inside)."""
    out = {}
    for k, floor in QUANTITIES:
        a = np.asarray([r[k] for r in mixed], dtype=np.float64)
        b = np.asarray([r[k] for r in fp64], dtype=np.float64)
        d = a - b
        m = 0.5 * (a.mean(0) + b.mean(0))
        se = d.std(0, ddof=1) / np.sqrt(len(d))
        keep = (np.abs(m) > floor) & (se > 0)
        z = d.mean(0)[keep] / se[keep]
        detect = 3.0 * se[keep] / np.abs(m[keep])
        excess = np.maximum(np.abs(d.mean(0)[keep]) - rel_tol * np.abs(m[keep]), 0.0) / se[keep]
        out[k] = dict(n=int(z.size), max_abs_z=float(np.abs(z).max()) if z.size else 0.0,
                      mean_z2=float((z ** 2).mean()) if z.size else 0.0,
                      max_excess_z=float(excess.max()) if z.size else 0.0,
                      max_rel_bias=float((np.abs(d.mean(0)[keep]) / np.abs(m[keep])).max()) if z.size else 0.0,
                      detectable_bias_median=float(np.median(detect)) if z.size else 0.0,
                      detectable_bias_max=float(detect.max()) if z.size else 0.0,
                      detectable_bias_min=float(detect.min()) if z.size else 0.0)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--cells", type=int, nargs=2, default=(128, 128))
    ap.add_argument("--ppc", type=int, default=100)
    ap.add_argument("--burn-in", type=int, default=None)
    ap.add_argument("--sample-every", type=int, default=20)
    ap.add_argument("--out", default="longrun.json")
    args = ap.parse_args()
    res = {"mixed": [], "fp64": [], "seconds": []}
    summary = None
    # seed by seed, both precisions, so that an interrupted run still leaves complete pairs in the output file
    for s in range(args.seeds):
        for prec, name in ((PREC_MIXED, "mixed"), (PREC_FP64, "fp64")):
            t0 = time.perf_counter()
            res[name].append(run(prec, 1000 + s, args.steps, tuple(args.cells), args.ppc, burn_in=args.burn_in,
                                 sample_every=args.sample_every))
            res["seconds"].append([name, s, time.perf_counter() - t0])
        summary = dict(config=dict(seeds=s + 1, steps=args.steps, cells=list(args.cells), ppc=args.ppc,
                                   burn_in=args.burn_in or args.steps // 2, sample_every=args.sample_every,
                                   samples=res["mixed"][0]["samples"]),
                       ion_flux=dict(mixed=np.mean([r["ion_flux"] for r in res["mixed"]], 0).tolist(),
                                     fp64=np.mean([r["ion_flux"] for r in res["fp64"]], 0).tolist()))
        if s >= 1:
            summary["paired"] = compare_paired(res["mixed"], res["fp64"])
            summary["welch"] = compare(res["mixed"], res["fp64"])
        with open(args.out, "w") as f:
            json.dump(dict(summary=summary, runs=res), f)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
