"""Benchmark of the SCF hot path: one Fock (G-matrix) build per step.

Workload (one step): the RHF two-electron Fock build G = 2J[P] - K[P] of
water with the s/p/d/f even-tempered basis plus the ghost-centre positron
s/p/d shells (87 shells, 292 Cartesian functions, 7,328,706 unique shell
quartets before Schwarz screening at 1e-14), from a seeded symmetric
density.  Every step recomputes every surviving integral (integral-direct)
and digests it into G.

Metric: shell quartets per second of the Fock build (whole job), and
seconds per SCF-iteration Fock build.  With --gpus N (torchrun) each rank
owns every N-th quartet of each class, builds its partial accumulator and
the partials are summed with one NCCL all-reduce before the symmetrising
finish (the reference's MPI_Reduce of G, rhfscf_mpi.c:36).

--impl reference times the reference's own CPU Fock build (oracle/_ref,
serial C, one core) on the same workload: the reference writes the ERIs to
disk once (untimed set-up) and each step digests one 1-GiB ERI file with
rhf_form_gmatrix (scfaux.c:429-552); its throughput is scaled to quartets
by the share of all integral records that file holds.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "water s/p/d/f + ghost positron s/p/d shells (87 shells, 292 functions), RHF Fock build"

# DRAM bytes (read + write) of the 55 class kernels and the unpack/finish
# kernels of one Fock build of this workload, from one ncu capture of
# dram__bytes_read.sum and dram__bytes_write.sum (cold caches per launch,
# the tuner's choices of a normal run replayed); the capture's command and
# per-kernel figures are kept with the other ncu summaries under profiles/.
STEP_DRAM_BYTES = 114.6e6
STEP_DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum over the 57 launches of one Fock build "
                    "(103.1 MB read, 58 MB of it the compacted quartet lists; 11.5 MB written, lane-kernel "
                    "spills of d/f classes), tuner choices replayed with PATGPU_TUNE_LOAD")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="patgpu", choices=["patgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tau", type=float, default=1e-14)
    ap.add_argument("--tau-fp32", type=float, default=1e-8,
                    help="Schwarz bound below which the mixed-precision leg runs quartets in FP32")
    ap.add_argument("--batch-molecules", type=int, default=32,
                    help="molecules in the batched (lock-step, graph-captured) leg; 0 skips it")
    ap.add_argument("--batch-max-atoms", type=int, default=8,
                    help="molecule sizes of the batched leg are uniform in 3..this")
    ap.add_argument("--alkane-carbons", type=int, default=12)
    ap.add_argument("--scf-maxit", type=int, default=50, help="SCF-iteration leg: iteration cap of both forms")
    ap.add_argument("--scf-tau-inc", type=float, default=1e-11,
                    help="SCF-iteration leg: density screening of the mixed batch's difference builds")
    ap.add_argument("--scf-tau-rel", type=float, default=1e-6,
                    help="SCF-iteration leg: screening of the mixed batch's builds at this times the largest DIIS "
                         "error, clipped to [--scf-tau-inc, --scf-tau-max] (0: fixed --scf-tau-inc)")
    ap.add_argument("--scf-tau-max", type=float, default=1e-7)
    ap.add_argument("--scf-ediis", type=int, default=1,
                    help="SCF-iteration leg: 1 blends energy-DIIS into DIIS while the DIIS error is above 1e-4")
    ap.add_argument("--scf-molecules", type=int, default=8,
                    help="molecules of the SCF-iteration leg (config-3 recipe); 0 skips it")
    ap.add_argument("--scf-max-atoms", type=int, default=24,
                    help="molecule sizes of the SCF-iteration leg are uniform in 3..this")
    ap.add_argument("--scf-level-shift", type=float, default=0.3,
                    help="SCF-iteration leg: virtual level shift (Eh) while the DIIS error exceeds 1e-3")
    ap.add_argument("--scf-full-every", type=int, default=8,
                    help="SCF-iteration leg: full Fock build every this many iterations of the mixed batch")
    ap.add_argument("--scf-tau-full", type=float, default=1e-14,
                    help="SCF-iteration leg: density screening of the mixed batch's full builds (0: none)")
    ap.add_argument("--no-organic40", action="store_true", help="skip the 40-atom (config-2) leg")
    ap.add_argument("--scf-iters", type=int, default=3,
                    help="alkane_dpm: SCF iterations before the gradient (timing; the converged "
                         "finite-difference check runs at C3H8 size in the GPU tests)")
    ap.add_argument("--workload", default="water_positron",
                    choices=["water_positron", "organic40", "alkane_dpm", "batch"],
                    help="water_positron: the headline line; organic40: FP64 vs mixed Fock build of the "
                         "40-atom organic molecule; alkane_dpm: SCF and analytic gradient of C12H26 with "
                         "positron shells and DPM (one GPU); batch: the batched leg alone")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=sorted(reasons), samples=len(rows))
        return out


# ------------------------------------------------------------- reference
def reference_fock(steps: int, warmup: int):
    """The reference's own Fock build on the host (see module docstring)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import patref   # CPU-baseline leg: the reference binary and its runner
    from patmol_b200 import configs, workload
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return None, "oracle/_ref/ref_harness was not built"
    b = configs.water_spdf_positron()
    qtotal = sum(workload.quartet_class_counts(b).values())
    with tempfile.TemporaryDirectory(prefix="patref_bench_") as d:
        b.write_patin(os.path.join(d, "patin.dat"))
        r = subprocess.run([harness, "bench1", str(steps), str(warmup)], cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            return None, "reference harness failed: " + r.stderr[-300:].replace("\n", " ")
        res = json.loads(r.stdout.strip().splitlines()[-1])
    frac = res["file_records"] / res["records"]
    t = res["gmat_seconds_per_call"]
    qps = qtotal * frac / t
    return {"value": qps, "unit": "quartets/s", "cores": 1, "kind": "reference",
            "sample": (f"reference rhf_form_gmatrix over one 1-GiB ERI file ({res['file_records']} of "
                       f"{res['records']} records, scaled to {qtotal} quartets); {t:.3f} s per file; "
                       f"ERI generation {res['eri_seconds']:.1f} s untimed"),
            "s_per_fock_build": t / frac, "eri_seconds": res["eri_seconds"]}, None


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    res, err = reference_fock(a.steps, a.warmup)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    line = {"metric": "ERI quartets/s (Fock build)", "value": res["value"], "unit": "quartets/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": res["s_per_fock_build"] * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "density": "seeded"},
            "impl": "reference", "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# --------------------------------------------------------------- batched
def batched_leg(a, torch, stream, nmol: int):
    """Lock-step Fock builds of many molecules as one CUDA graph (patgpu_batch)
    against the same builds launched molecule by molecule, FP64 and mixed."""
    import numpy as np
    from patmol_b200 import configs, gpu
    rng = np.random.default_rng(77)
    sizes = rng.integers(3, a.batch_max_atoms + 1, size=nmol)   # uniform in 3..max atoms
    bases = [configs.organic_basis(int(k), 1000 + i, with_f=False) for i, k in enumerate(sizes)]
    gbs = [gpu.GpuBasis(bb, schwarz_tau=a.tau) for bb in bases]
    batch = gpu.GpuBatch(gbs)
    Ps = [np.random.default_rng(2000 + i).normal(scale=0.05, size=g.no2) for i, g in enumerate(gbs)]
    G64 = batch.rhf_form_gmatrix(Ps)                # loads P into the batch buffers, captures the graph
    sh = stream.cuda_stream
    bufs = [batch.buffers(m) for m in range(nmol)]

    def timed(fn, reps):
        for _ in range(max(a.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def sequential():
        for g, (dP, dG) in zip(gbs, bufs):
            g.rhf_gmatrix_device(dP, dG, sh)

    reps = max(1, min(a.steps, 5))
    t_graph = timed(lambda: batch.launch(sh), reps)
    t_seq = timed(sequential, reps)
    st = batch.stats()
    batch.set_mixed_precision(a.tau_fp32)
    Gmx = batch.rhf_form_gmatrix(Ps)
    t_mixed = timed(lambda: batch.launch(sh), reps)
    stm = batch.stats()
    dG = max(float(np.abs(x - y).max()) for x, y in zip(Gmx, G64))
    batch.close()
    for g in gbs:
        g.close()
    q = st["quartets"]
    return {"workload": f"{nmol} seeded organic molecules (C/N/O/H walk), 3-{a.batch_max_atoms} atoms uniform, "
                        "config-0 s/p/d basis, RHF Fock build of every molecule per step",
            "molecules": nmol, "basis_functions": int(sum(bb.norb for bb in bases)), "quartets": q,
            "graph_nodes": st["graph_nodes"],
            "l2": (f"not flushed: each step reads {8 * q / 1e9:.1f} GB of compacted quartet lists (8 B per "
                   "quartet), far above the 126 MB L2"),
            "ms_per_step_graph": t_graph, "ms_per_step_sequential": t_seq,
            "quartets_per_s_graph": q / (t_graph * 1e-3), "speedup_graph_vs_sequential": t_seq / t_graph,
            "mixed": {"tau_fp32": a.tau_fp32, "fp32_quartets": stm["fp32_quartets"], "ms_per_step": t_mixed,
                      "speedup_vs_fp64_graph": t_graph / t_mixed, "max_abs_dG_vs_fp64": dG}}


# ------------------------------------------------------------ SCF leg
def scf_leg(torch):
    """Water s/p/d (132 functions): full SCF to 1e-12 Eh through the GPU Fock
    build, with full builds every iteration and with incremental
    (density-difference, density-screened) builds; wall time per iteration
    includes the host diagonalisation."""
    from patmol_b200 import configs, gpu, scf
    b = configs.water_spd()
    out = {"workload": "water s/p/d (51 shells, 132 functions), RHF to 1e-12 Eh, DIIS"}
    for name, inc in (("full", False), ("incremental", True)):
        g = gpu.GpuBasis(b)
        torch.cuda.synchronize()
        t0 = time.time()
        r = scf.rhf(b, gpu=g, incremental=inc)
        dt = time.time() - t0
        out[name] = {"energy": r.energy, "iterations": r.iterations, "converged": r.converged,
                     "seconds": dt, "s_per_iteration": dt / max(r.iterations, 1)}
        if inc:
            out[name]["quartets_per_iteration"] = r.quartets_computed
        g.close()
    out["dE_incremental_vs_full"] = out["incremental"]["energy"] - out["full"]["energy"]
    return out


def scf_iteration_leg(a, torch):
    """Batched-SCF throughput (the metric's s/SCF-iteration on the config-3
    recipe): a seeded sample of molecules of 3..max atoms (C/N/O/H walk,
    config-0 s/p/d basis) converged two ways:
      plain: one molecule after the other, every iteration a full FP64 Fock
             build (patgpu_rhf_gmatrix);
      mixed: all molecules in lock step, one CUDA-graph launch per iteration
             (patgpu_batch), FP32 window (term bound below tau_fp32) in every
             build, density-screened difference builds (tau_inc) between full
             builds every full_every iterations, density-weighted FP32 while
             the density still moves (the final iterations' difference
             builds stay FP64), converged molecules skipped; every build's
             screening threshold follows the SCF: tau_rel times the largest
             DIIS error still iterating, clipped to [tau_inc, tau_max]; the
             final energies come from unscreened builds.
    Both use DIIS with energy-DIIS blended in while the DIIS error is above
    1e-4, a 0.3 Eh virtual level shift while it is above 1e-3, the device
    eigensolver and canonical orthogonalisation over
    overlap eigenvalues above 1e-7 (the diffuse 0.08 s exponents on atoms
    2.6-2.9 bohr apart make the overlap nearly singular), converged at
    |dE| < 1e-8 Eh, max|FPS-SPF| < 1e-5, max|dP| < 1e-5, at most scf_maxit
    iterations.  Some walk geometries (stretched bonds to H) are
    near-degenerate and do not converge in RHF within the cap in either
    form; they count with their capped iterations.  Reported: SCF
    iterations per second of the Fock builds (device-timed; the metric) and
    of the whole SCF (wall, host steps included), the Fock time to finish
    every molecule, and |E_mixed - E_plain| of every molecule converged in
    both forms."""
    import numpy as np
    from patmol_b200 import configs, scf
    rng = np.random.default_rng(303)
    sizes = rng.integers(3, a.scf_max_atoms + 1, size=a.scf_molecules)
    bases = [configs.organic_basis(int(k), 3000 + i, with_f=False) for i, k in enumerate(sizes)]
    kw = dict(conv=1e-8, comm_tol=1e-5, dp_tol=1e-5, maxit=a.scf_maxit, smin=1e-7, device_linalg=True,
              level_shift=a.scf_level_shift, shift_tol=1e-3, ediis=bool(a.scf_ediis))
    mix = dict(tau_fp32=a.tau_fp32, incremental=True, tau_inc=a.scf_tau_inc, tau_inc32=1e-6,
               full_every=a.scf_full_every, tau_full=a.scf_tau_full, tau_rel=a.scf_tau_rel, tau_max=a.scf_tau_max)
    torch.cuda.synchronize()
    t0 = time.time()
    plain = [scf.rhf(b, **kw) for b in bases]
    t_plain = time.time() - t0
    it_plain = sum(r.iterations for r in plain)
    fock_plain = sum(r.fock_seconds for r in plain)
    computed, fock_b = [], []
    t0 = time.time()
    mixed = scf.rhf_batch(bases, computed=computed, fock_seconds=fock_b, **mix, **kw)
    t_mixed = time.time() - t0
    it_mixed = sum(r.iterations for r in mixed)
    fock_mixed = sum(fock_b)
    both = [i for i, (x, y) in enumerate(zip(plain, mixed)) if x.converged and y.converged]
    dE = {i: abs(plain[i].energy - mixed[i].energy) for i in both}
    return {"workload": f"{a.scf_molecules} seeded molecules of 3-{a.scf_max_atoms} atoms (C/N/O/H walk), config-0 "
                        "s/p/d basis, RHF converged to dE < 1e-8 Eh, max|FPS-SPF| < 1e-5, max|dP| < 1e-5",
            "atoms": [int(x) for x in sizes], "basis_functions": [b.norb for b in bases],
            "max_iterations": a.scf_maxit, "level_shift": a.scf_level_shift,
            "plain_fp64": {"wall_s": t_plain, "fock_s": fock_plain, "iterations": it_plain,
                           "fock_s_per_scf_iteration": fock_plain / it_plain,
                           "wall_s_per_scf_iteration": t_plain / it_plain,
                           "converged": int(sum(r.converged for r in plain)),
                           "iterations_per_molecule": [r.iterations for r in plain],
                           "fock_s_per_molecule": [r.fock_seconds for r in plain]},
            "mixed_batched": {"wall_s": t_mixed, "fock_s": fock_mixed, "iterations": it_mixed,
                              "fock_s_per_scf_iteration": fock_mixed / it_mixed,
                              "wall_s_per_scf_iteration": t_mixed / it_mixed,
                              "converged": int(sum(r.converged for r in mixed)),
                              "lockstep_iterations": len(computed),
                              "iterations_per_molecule": [r.iterations for r in mixed],
                              "quartets_per_build": computed, "fock_s_per_build": fock_b, **mix},
            "scf_iteration_speedup_fock": (it_mixed / fock_mixed) / (it_plain / fock_plain),
            "scf_iteration_speedup_wall": (it_mixed / t_mixed) / (it_plain / t_plain),
            "time_to_solution_speedup_fock": fock_plain / fock_mixed,
            "converged_in_both": len(both),
            "max_abs_dE_converged": max(dE.values()) if dE else None,
            "dE_per_converged_molecule": {str(i): v for i, v in dE.items()}}


def linalg_leg():
    """The SCF step after the Fock build (X^T F X, eigenpairs, C = X V,
    P = C_occ C_occ^T, W) at the largest config-3 molecule's size (1056
    functions) and at config 2's (2560): the GPU (patgpu_scf_density_host,
    host buffers in and out) against numpy on the host (threads as numpy
    uses them).  Seeded symmetric F, X = 1."""
    import numpy as np
    from patmol_b200 import gpu
    out = {"workload": "SCF density step, seeded symmetric F, X = identity, nocc = n/8"}
    for n in (1056, 2560):
        rng = np.random.default_rng(n)
        A = rng.normal(size=(n, n))
        F = (A + A.T) / 2
        il = np.tril_indices(n)
        Fp = F[il].copy()
        X = np.eye(n)
        nocc = n // 8
        t0 = time.time()
        e, V = np.linalg.eigh(X.T @ F @ X)
        C = X @ V
        P = C[:, :nocc] @ C[:, :nocc].T
        W = (C[:, :nocc] * e[:nocc]) @ C[:, :nocc].T
        t_host = time.time() - t0
        la = gpu.GpuScfLinalg(X, nocc)
        la.density(Fp)                       # warm-up
        t0 = time.time()
        eg, _, Pg, Wg = la.density(Fp)
        t_dev = time.time() - t0
        la.close()
        out[str(n)] = {"host_s": t_host, "gpu_s": t_dev, "speedup": t_host / t_dev,
                       "max_abs_dP": float(np.abs(Pg - P[il]).max()), "max_abs_deps": float(np.abs(eg - e).max())}
    return out


# ------------------------------------------------------ other workloads
def _timed_builds(torch, stream, G, P, Gd, reps):
    """Device-timed Fock builds (ms each) through patgpu_rhf_gmatrix_device."""
    sh = stream.cuda_stream
    G.rhf_gmatrix_device(P.data_ptr(), Gd.data_ptr(), sh)
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        G.rhf_gmatrix_device(P.data_ptr(), Gd.data_ptr(), sh)
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return sum(out) / len(out)


def organic40_leg(a, torch, stream):
    """Config: 40-atom seeded organic molecule (C/N/O/H walk), s/p/d/f basis;
    FP64 vs mixed (Schwarz bound < tau_fp32 in FP32) Fock builds at the core
    Hamiltonian guess density, with the energy change tr(P dG)."""
    import numpy as np
    from patmol_b200 import configs, gpu, workload
    from patmol_b200.basis import unpack
    from patmol_b200.scf import orthogonalizer
    t0 = time.time()
    b = configs.organic_basis(40, 2, with_f=True)
    G = gpu.GpuBasis(b, schwarz_tau=a.tau)
    G.two_electron_ints()
    t_setup = time.time() - t0
    st = G.stats()
    Sp, _, Hp = G.one_electron_ints()
    n = b.norb
    X = orthogonalizer(unpack(Sp, n))
    e, V = np.linalg.eigh(X.T @ unpack(Hp, n) @ X)
    C = X @ V
    Pf = C[:, :b.nelec // 2] @ C[:, :b.nelec // 2].T
    Pp = Pf[np.tril_indices(n)]
    il = np.tril_indices(n)
    w = np.where(il[0] == il[1], 1.0, 2.0)
    P = torch.from_numpy(Pp.copy()).to("cuda")
    Gd = torch.empty_like(P)
    reps = max(1, min(a.steps, 1))
    ms64 = _timed_builds(torch, stream, G, P, Gd, reps)
    G64 = Gd.cpu().numpy()
    nfp32 = G.set_mixed_precision(a.tau_fp32)
    msmx = _timed_builds(torch, stream, G, P, Gd, reps)
    Gmx = Gd.cpu().numpy()
    flops = workload.fock_flops(G.class_counts(), "rhf")
    kern_ns, _ = G.last_timing()
    q = st["quartets"]
    return {"metric": "ERI quartets/s (Fock build)", "value": q / (ms64 * 1e-3), "unit": "quartets/s",
            "n_gpus": 1, "steps": reps, "warmup": 1, "ms_per_step": ms64, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "40-atom seeded organic molecule (C/N/O/H walk, seed 2), s/p/d/f "
                                   "even-tempered basis, RHF Fock build at the core-Hamiltonian guess density",
                       "basis_functions": n, "shells": b.nshell, "quartets": q,
                       "quartets_unscreened": st["unscreened"], "schwarz_tau": a.tau,
                       "setup_s": t_setup},
            "roofline": {"bound": "fp64", "achieved": flops / (ms64 * 1e-3) / 1e12, "unit": "TFLOP/s",
                         "peak": gpu.fp64_peak_tflops()},
            "mixed": {"tau_fp32": a.tau_fp32, "fp32_quartets": nfp32, "ms_per_step": msmx,
                      "speedup_vs_fp64": ms64 / msmx,
                      "dE_fixed_density": float(np.sum(w * Pp * (Gmx - G64))),
                      "max_abs_dG_vs_fp64": float(np.abs(Gmx - G64).max())}}


def alkane_dpm_leg(a, torch, stream):
    """Config: C12H26 (seeded jitter), s/p/d basis, ghost centroid with the
    positron s/p/d shells and DPM on; converged SCF, then the analytic
    gradient (derivative ERIs recomputed, not stored)."""
    import numpy as np
    from patmol_b200 import configs, gpu, scf
    from patmol_b200.basis import Basis
    sym, xyz = configs.alkane(a.alkane_carbons, 0)
    mol = configs.molecule_basis(sym, xyz, with_f=False)
    cen = xyz.mean(axis=0)
    specs = [(r[1], r[2], r[3], r[4]) for r in mol.raw] + configs.ghost_shells(len(sym))
    q = np.concatenate([mol.charges, [0.0]])
    b = Basis.from_shell_list(q, np.vstack([xyz, cen[None, :]]), specs, nelec=mol.nelec, mult=1,
                              dpm=1).dpm_augmented(cen)
    t0 = time.time()
    G = gpu.GpuBasis(b, schwarz_tau=a.tau)
    t_setup = time.time() - t0
    t0 = time.time()
    res = scf.rhf(b, dpm=True, gpu=G, conv=1e-10, maxit=a.scf_iters)
    t_scf = time.time() - t0
    ns_fock, _ = G.last_timing()
    torch.cuda.synchronize()
    t0 = time.time()
    g = G.rhf_gradient(res.P, res.W, parts=G.GRAD_ALL, with_dpm=True)
    t_grad = time.time() - t0
    t0 = time.time()
    g2 = G.rhf_gradient(res.P, res.W, parts=G.GRAD_2E)
    t_grad2e = time.time() - t0
    st = G.stats()
    torque = np.cross(b.coords, g).sum(axis=0)
    return {"metric": "analytic gradient (s)", "value": t_grad, "unit": "s", "n_gpus": 1, "steps": 1,
            "warmup": 0, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"C{a.alkane_carbons}H{2 * a.alkane_carbons + 2} (C-C 2.91, C-H 2.06 bohr, "
                                   "seeded 0.05 bohr jitter), s/p/d basis, ghost centroid with positron s/p/d "
                                   f"shells, DPM on, RHF; gradient at the density after {a.scf_iters} SCF "
                                   "iterations (timing)",
                       "basis_functions": b.norb, "shells": b.nshell, "quartets": st["quartets"],
                       "quartets_unscreened": st["unscreened"], "schwarz_tau": a.tau, "setup_s": t_setup},
            "scf": {"energy": res.energy, "iterations": res.iterations, "converged": res.converged,
                    "seconds": t_scf, "last_fock_build_ms": ns_fock / 1e6},
            "gradient": {"seconds_all_parts": t_grad, "seconds_two_electron": t_grad2e,
                         "max_abs": float(np.abs(g).max()), "net_force": float(np.abs(g.sum(axis=0)).max()),
                         "net_torque": float(np.abs(torque).max()),
                         "positron_centre": [float(x) for x in g[b.skipcen]],
                         "two_electron_share_max_abs": float(np.abs(g2).max())}}


# ------------------------------------------------------------------- GPU
def main():
    a = parse()
    if a.impl == "reference":
        run_reference_arm(a)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    from patmol_b200 import configs, gpu, workload
    if a.workload != "water_positron":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        if a.workload == "batch":
            out = batched_leg(a, torch, stream, max(a.batch_molecules, 1))
            out.update(metric="ERI quartets/s (batched Fock build)", value=out["quartets_per_s_graph"],
                       unit="quartets/s", n_gpus=1, steps=max(1, min(a.steps, 5)), warmup=max(a.warmup, 1),
                       higher_is_better=True, dtype="f64", data="synthetic")
            print(json.dumps(out))
            return
        leg = organic40_leg if a.workload == "organic40" else alkane_dpm_leg
        print(json.dumps(leg(a, torch, stream)))
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream

    b = configs.water_spdf_positron()
    n = b.norb
    no2 = n * (n + 1) // 2
    G = gpu.GpuBasis(b, schwarz_tau=a.tau)
    G.two_electron_ints(0, rank, world)
    st = G.stats()
    counts = G.class_counts()
    my_flops = workload.fock_flops(counts, "rhf")
    my_q = st["quartets"]
    tot = torch.tensor([my_q, my_flops], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tot)
    total_q, total_flops = int(tot[0].item()), float(tot[1].item())

    rng = np.random.default_rng(1234)
    P_host = torch.from_numpy(rng.normal(scale=0.05, size=no2)).pin_memory()
    G_host = torch.empty(no2, dtype=torch.float64).pin_memory()
    P = P_host.to(dev)
    # accumulator: n*n pairs of int64 words with exact fixed-point accumulation
    # (summed as integers across ranks), n*n doubles with FP64 atomics
    det = G.accumulator_bytes() == 16 * n * n
    A = torch.empty(G.accumulator_bytes() // 8, dtype=torch.int64 if det else torch.float64, device=dev)
    Gd = torch.empty(no2, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    def step():
        G.rhf_accumulate_device(P.data_ptr(), A.data_ptr(), sh)
        if world > 1:
            dist.all_reduce(A)
        G.finish_gmatrix_device(A.data_ptr(), Gd.data_ptr(), sh)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    kern_ns = 0.0
    launches = 0
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    for i in range(a.steps):
        flush.fill_(float(i))                      # evict L2 between steps (not timed)
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
        torch.cuda.synchronize()
        kns, nl = G.last_timing()
        kern_ns += kns
        launches += nl + 2                        # class kernels + unpack + finish
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / a.steps
    kern_ms = kern_ns / 1e6 / a.steps

    # end to end through the public C ABI: pinned host P in, host G out
    e2e_ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_ev[0].record(stream)
    for i in range(a.steps):
        P.copy_(P_host, non_blocking=True)
        step()
        G_host.copy_(Gd, non_blocking=True)
    e2e_ev[1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2e_ev[0].elapsed_time(e2e_ev[1]) / a.steps
    clk = clocks.stop()

    # mixed-precision leg: the same Fock builds with FP32 arithmetic for the
    # quartets whose Schwarz bound is below tau_fp32 (FP64 accumulation)
    ref_G = Gd.clone()
    nfp32 = G.set_mixed_precision(a.tau_fp32)
    for _ in range(a.warmup):
        step()
    mx_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    for i in range(a.steps):
        flush.fill_(float(i))
        mx_ev[i][0].record(stream)
        step()
        mx_ev[i][1].record(stream)
        torch.cuda.synchronize()
    mixed_ms = sum(e0.elapsed_time(e1) for e0, e1 in mx_ev) / a.steps
    dG = (Gd - ref_G).abs().max().item()
    G.set_mixed_precision(0.0)
    nfp32_t = torch.tensor([float(nfp32)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(nfp32_t)

    t = torch.tensor([step_ms, e2e_ms, kern_ms, mixed_ms, dG], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms, e2e_ms, kern_ms, mixed_ms, dG = (float(x) for x in t.tolist())

    line = None
    if rank == 0:
        peak = gpu.fp64_peak_tflops()
        dmma = gpu.dmma_peak_tflops()
        achieved = my_flops / (kern_ms * 1e-3) / 1e12 if kern_ms > 0 else None
        line = {
            "metric": "ERI quartets/s (Fock build)",
            "value": total_q / (step_ms * 1e-3),
            "unit": "quartets/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": step_ms,
            "s_per_scf_iteration_fock": step_ms * 1e-3,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "quartets": total_q, "quartets_unscreened": st["unscreened"],
                       "schwarz_tau": a.tau, "basis_functions": n, "density": "seeded N(0,0.05^2)",
                       "l2": "flushed between steps (256 MB write, untimed)",
                       "parallelism": f"quartet split x{world}" + (" + NCCL all-reduce" if world > 1 else "")},
            "e2e": {"value": total_q / (e2e_ms * 1e-3), "unit": "quartets/s",
                    "h2d_bytes_per_step": no2 * 8, "d2h_bytes_per_step": no2 * 8,
                    "path": "pinned P -> patgpu_rhf_accumulate_device -> patgpu_finish_gmatrix_device -> pinned G"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": STEP_DRAM_BYTES,
                         "traffic_source": STEP_DRAM_SOURCE,
                         "peak_source": "measured FP64 FMA probe (patgpu_fp64_peak), this GPU, this run",
                         "fp64_mma_tflops": dmma,
                         "fp64_mma_source": "measured mma.sync m8n8k4 FP64 probe (patgpu_dmma_peak), this GPU, "
                                            "this run: the only FP64 tensor-core path on sm_100a",
                         "algorithmic_flops_per_step": my_flops,
                         "kernel_ms_per_step": kern_ms},
            "mixed": {"tau_fp32": a.tau_fp32, "fp32_quartets": int(nfp32_t.item()),
                      "ms_per_step": mixed_ms, "speedup_vs_fp64": step_ms / mixed_ms,
                      "max_abs_dG_vs_fp64": dG},
            "gpu_launches": launches,
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        if world == 1 and a.batch_molecules > 0:
            line["batched"] = batched_leg(a, torch, stream, a.batch_molecules)
        if world == 1:
            line["scf"] = scf_leg(torch)
            line["linalg"] = linalg_leg()
            if not a.no_organic40:
                o = organic40_leg(a, torch, stream)
                line["organic40"] = {"workload": o["config"]["workload"], "basis_functions": o["config"]["basis_functions"],
                                     "quartets": o["config"]["quartets"], "ms_per_fock_build_fp64": o["ms_per_step"],
                                     "quartets_per_s_fp64": o["value"], "roofline": o["roofline"], "mixed": o["mixed"],
                                     "setup_s": o["config"]["setup_s"]}
            if a.scf_molecules > 0:
                line["scf_iteration"] = scf_iteration_leg(a, torch)
        if world == 1 and not a.no_cpu_baseline:
            res, err = reference_fock(2, 1)
            line["cpu_baseline"] = ({k: res[k] for k in ("value", "unit", "cores", "kind", "sample")}
                                    if res else {"unavailable": err})
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
