"""Benchmark: Gauss-point updates/s of the explicit SMA (law 160) step.

Workload (one GPU): NiTi cylinder r = 5 mm, L = 50 mm, HEX08 O-grid of
1,998,848 elements (2,034,729 nodes, 16.0 M Gauss points), interior nodes
jittered U(-0.1,0.1)h, a material per element (E_A, E_M, eps_L and the four
transformation stresses sampled +-10 % from a seed), temperature 300-320 K
shifting the transformation stresses by 6.5 MPa/K, x = 0 clamped, x = L
pushed to -3 % axial strain and released with smooth steps; central
difference at dt = 0.5 dt_crit, prestrained 1 % so the return map is live.
A step is one pass of the explicit scheme over the whole mesh (element loop
+ nodal update, BCs and time advanced on the device).  `value` times the
FP32 precision form (FP32 kinematics and constitutive update, FP64 return
map, force accumulation and integration); the plain FP64 form runs the same
steps from the same start beside it, and `error_vs_fp64` compares the two
at the end of the timed window (Gauss-point stress, displacement, martensite
fraction, reaction on the pushed face).  --workload cantilever (640 k
elements, tip traction) and ensemble (256 specimens) select the others.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp32|fp64] [--scatter atomic|color]

--gpus N > 1 (under torchrun): the cylinder and the cantilever are split
into N element slabs, one per rank, the interface rows exchanged with the
neighbouring slabs every step while the interior elements compute (strong
scaling; --no-partition runs one replica per rank instead); --workload
ensemble shards its 256 specimens across the ranks, largest first onto the
least loaded rank, with no exchange (strong scaling).  The time is the
maximum over ranks of the device time.
--impl reference times the CPU restatement of the reference path (the
oracle: the reference is Fortran and cannot be built here) on the host
cores of rank 0, on a bounded sample of the same workload.
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

WORKLOADS = {"cantilever": "cantilever_400x40x40_hex08",
             "cylinder": "cylinder_ogrid_2.0M_hex08_per_element_materials",
             "ensemble": "ensemble_256_specimens_hex08"}


L2_BYTES = 126e6          # B200 L2


def arm_config(args, world, nelem, npoin, gauss_points, wset_mesh):
    """The workload the line is quoted on -- the same dict in the reference
    arm's line as in this arm's: the mesh (nelem, npoin of the job's unique
    mesh or meshes), its Gauss points over the whole job, the form, the
    prestrain, the working set per GPU against L2 and how the job uses the
    GPUs.  How this arm launches it (threads per block, scatter, tuning) is
    in the line's `launch`."""
    sharded = args.workload == "ensemble" and world > 1
    split = bool(args.partition) and not sharded
    per_gpu = wset_mesh / world if (sharded or split) else wset_mesh
    if sharded:
        par = f"specimens sharded over {world} GPUs (no exchange)"
    elif split:
        par = (f"one mesh in {world} element slabs, the shared nodes' residual rows exchanged with the "
               "neighbouring slabs every step, overlapped with the interior elements")
    else:
        par = f"replicas x{world}" if world > 1 else "single GPU"
    return {"workload": workload_name(args.workload, args.div), "nelem": int(nelem), "npoin": int(npoin),
            "gauss_points": int(gauss_points), "precision": args.precision, "prestrain": args.prestrain,
            "l2": (("working set > L2 (state, nodal arrays and connectivity "
                    f"~{per_gpu / 1e6:.0f} MB per step per GPU vs 126 MB L2)") if per_gpu > L2_BYTES else
                   (f"working set ~{per_gpu / 1e6:.0f} MB per GPU fits the 126 MB L2 (a test-sized mesh: "
                    "its arrays stay cached between steps)")),
            "parallelism": par}


def working_set(prob, precision):
    """Bytes one step streams: the element kernel's algorithmic bytes and the
    nodal update's six FP64 nodal arrays read and written."""
    return algorithmic_bytes(prob, precision) + 6 * 24 * prob.npoin


def workload_name(workload, div):
    """The workload's name as run: --div coarsens the cantilever and the
    cylinder by that factor per direction and cuts the ensemble to 256 / div
    specimens."""
    if div == 1:
        return WORKLOADS[workload]
    if workload == "ensemble":
        return f"ensemble_{max(2, 256 // div)}_specimens_hex08"
    return f"{WORKLOADS[workload]}_coarsened_{div}x"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "surrogate"],
                    help="the timed form: fp32 (FP32 kinematics and law, FP64 return map and integration), "
                         "fp64, or surrogate (the fp32 form with the learned surrogate in its element loop)")
    ap.add_argument("--scatter", default="atomic", choices=["atomic", "color"])
    ap.add_argument("--no-extras", action="store_true", help="skip fp64/e2e/cpu legs")
    ap.add_argument("--div", type=int, default=1, help="coarsen the mesh (tests only)")
    ap.add_argument("--prestrain", type=float, default=0.01,
                    help="initial axial strain (both arms): 1%% is just past the AS start")
    ap.add_argument("--workload", default="cylinder", choices=list(WORKLOADS),
                    help="cylinder (default: 2.0M-element O-grid, per-element materials, temperature "
                         "field), cantilever 400x40x40 or ensemble (256 specimens)")
    ap.add_argument("--layers", type=int, default=0,
                    help="cylinder only: axial element layers (0: the full 488); a shorter cylinder "
                         "is the profiling case of the same kernel")
    ap.add_argument("--write-profile", metavar="CSV", default=None,
                    help="turn `ncu -i <rep> --page raw --csv` output into the machine-read profile "
                         "summary of this precision/workload (profiles/k_element_<prec>_<workload>.json)")
    ap.add_argument("--surrogate", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the FP32 form with the learned surrogate (trained first, on the GPU)")
    ap.add_argument("--surrogate-samples", type=int, default=20_000_000, help="plain-law samples generated")
    ap.add_argument("--surrogate-epochs", type=int, default=4)
    ap.add_argument("--surrogate-gate", type=float, default=3.0, help="out-of-envelope score limit")
    ap.add_argument("--block", type=int, default=0, help="threads per element block (0: library default)")
    ap.add_argument("--autotune", action="store_true", help="pick block and scatter by timing candidates")
    ap.add_argument("--partition", action=argparse.BooleanOptionalAction, default=None,
                    help="split the one mesh over the ranks (element slabs, interface elements first; the "
                         "shared nodes' residual exchanged with the neighbouring slabs while the interior "
                         "elements compute): strong scaling.  Default: on for the cylinder and the "
                         "cantilever under --gpus N > 1, off at N = 1; the ensemble shards its specimens")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


class Clocks:
    """nvidia-smi sampler for the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append(dict(sm=float(f[1]), smax=float(f[2]), power=float(f[3]),
                                 hw=f[5], hwt=f[6], swt=f[7], swp=f[8]))
            except ValueError:
                continue
        if not rows:
            return None
        load = [r for r in rows if r["power"] > 250.0] or rows
        reasons = sorted({name for r in load for name, key in
                          (("hw_slowdown", "hw"), ("hw_thermal_slowdown", "hwt"),
                           ("sw_thermal_slowdown", "swt"), ("sw_power_cap", "swp"))
                          if r[key].lower().startswith("active")})
        return {"sm_mhz": statistics.median(r["sm"] for r in load),
                "sm_max_mhz": max(r["smax"] for r in rows), "reasons": reasons,
                "samples": len(rows), "samples_under_load": len(load)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


KERNEL_SOURCES = ("alya_sma_b200/csrc/sma_capi.cu", "alya_sma_b200/csrc/sma_kernels.cuh",
                  "alya_sma_b200/csrc/sma_law.cuh", "alya_sma_b200/csrc/sma_surrogate.cuh",
                  "alya_sma_b200/csrc/sma_surrogate_elem.cuh", "alya_sma_b200/build.py")


def kernel_source_hash():
    """Hash of the sources the element kernel is compiled from: a profile
    taken on another build of the kernel says nothing about this one."""
    import hashlib
    h = hashlib.sha256()
    for rel in KERNEL_SOURCES:
        path = os.path.join(ROOT, rel)
        if os.path.exists(path):
            with open(path, "rb") as fh:
                h.update(rel.encode() + b"\0" + fh.read())
    return h.hexdigest()[:16]


def profile_json(precision, workload):
    return os.path.join(ROOT, "profiles", f"k_element_{precision}_{workload}.json")


_UNITS = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12,
          "KB": 1e3, "MB": 1e6, "GB": 1e9, "inst": 1.0, "Kinst": 1e3, "Minst": 1e6, "Ginst": 1e9,
          "ns": 1e-9, "us": 1e-6, "usecond": 1e-6, "msecond": 1e-3, "nsecond": 1e-9, "ms": 1e-3,
          "": 1.0, "warp": 1.0}


def write_profile(csv_path, precision, workload, nelem, note=""):
    """Machine-read summary of one ncu capture (`ncu -i rep --page raw --csv`)
    of the element kernel: DRAM bytes and warp instructions per launch and
    the number of elements the captured launch processed, stamped with the
    hash of the kernel sources; written to profiles/ as JSON."""
    import csv
    with open(csv_path, newline="") as fh:
        rows = list(csv.reader(fh))
    head = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    names, units = rows[head], rows[head + 1]
    col = {n: i for i, n in enumerate(names)}

    def val(r, metric):
        if metric not in col:
            return None
        raw = r[col[metric]].replace(",", "")
        try:
            return float(raw) * _UNITS.get(units[col[metric]].strip(), 1.0)
        except ValueError:
            return None

    launches = [r for r in rows[head + 2:] if len(r) == len(names) and "k_element" in r[col["Kernel Name"]]]
    if not launches:
        raise SystemExit(f"no k_element launch in {csv_path}")
    n = len(launches)
    mean = lambda m: (sum(val(r, m) or 0.0 for r in launches) / n) if all(val(r, m) is not None for r in launches) else None
    rd, wr = mean("dram__bytes_read.sum"), mean("dram__bytes_write.sum")
    out = {"kernel": launches[0][col["Kernel Name"]], "precision": precision, "workload": workload,
           "elements_per_launch": int(nelem), "launches_captured": n,
           "dram_bytes_per_launch": (rd + wr) if rd is not None and wr is not None else None,
           "dram_read_bytes_per_launch": rd, "dram_write_bytes_per_launch": wr,
           "warp_inst_per_launch": mean("smsp__inst_executed.sum"),
           "duration_s_under_ncu": mean("gpu__time_duration.sum"),
           "registers_per_thread": mean("launch__registers_per_thread"),
           "kernel_source_hash": kernel_source_hash(), "note": note}
    path = profile_json(precision, workload)
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
        fh.write("\n")
    print(path)
    return out


def load_profile(precision, workload, nelem):
    """The machine-written ncu summary of the element kernel for this
    precision and workload, scaled from the captured launch's element count
    to `nelem` (traffic and instructions grow with the elements processed),
    or None when there is none or it was taken on other kernel sources."""
    try:
        with open(profile_json(precision, workload)) as fh:
            p = json.load(fh)
    except (OSError, ValueError):
        return None
    if p.get("kernel_source_hash") != kernel_source_hash():
        return None
    k = nelem / float(p["elements_per_launch"])
    return {"traffic": None if p.get("dram_bytes_per_launch") is None else p["dram_bytes_per_launch"] * k,
            "warp_inst": None if p.get("warp_inst_per_launch") is None else p["warp_inst_per_launch"] * k,
            "scaled_from_elements": p["elements_per_launch"], "sms": 148}


def per_element_values(prob):
    """Material values the element kernel needs per element: the seven the
    cylinder and the ensemble sample (E_A, E_M, eL, four transformation
    stresses) plus the temperature with per-element materials; the
    temperature alone with one material and a temperature field."""
    if len(prob.props) > 1:
        return 8
    return 1 if prob.tempe is not None else 0


def algorithmic_bytes(prob, precision):
    """Minimum HBM traffic of one element-kernel launch: connectivity, state
    read + write (3 words per Gauss point), the per-element material values
    and temperature (in the precision's word), one read of coordinates and
    displacements and one read-modify-write of the residual per node; with
    the surrogate also the held stress residual read (6 FP16 per Gauss
    point; its writes by the plain law's points and the network's inputs
    staged for 1/64 of the tiles are not counted)."""
    s = 8 if precision == "fp64" else 4
    held = 8 * 6 * 2 if precision == "surrogate" else 0
    return prob.nelem * (32 + 2 * 8 * 3 * s + held + per_element_values(prob) * s) + prob.npoin * (24 + 24 + 48)


def build_problem(workload, div, rank=0, world=1, layers=0):
    """The workload's mesh on this rank.  The ensemble shards its specimens
    across ranks (largest first onto the least loaded rank); the other
    workloads run one replica per rank.  layers > 0 shortens the cylinder to
    that many axial element layers (same cross-section and element size)."""
    from alya_sma_b200 import problem as P
    if workload == "cylinder":
        return P.cylinder_2m(nsteps=10000, div=div, layers=layers or None)
    if workload == "ensemble":
        # specimens concatenated by size, so each size bucket is one element
        # range (the autotuner's launch plan gives each its own block)
        nspec = max(2, 256 // div)
        if world > 1:
            from alya_sma_b200 import dist as D
            mine = D.shard_specimens(P.ensemble_sizes(nspec), rank, world)
            return P.ensemble(nspec=nspec, nsteps=5000, subset=mine, by_size=True)
        return P.ensemble(nspec=nspec, nsteps=5000, by_size=True)
    return P.cantilever_400x40x40(nsteps=20000, div=div)


# steps between two evaluations of the surrogate's network on a tile of 16
# elements (the library's default): ngp / SUR_PERIOD evaluations per step
SUR_PERIOD = 64


def compare_forms(prob, s32, s64, nsteps, spread=None):
    """Error of the FP32 precision form against the plain FP64 form after the
    same `nsteps` steps from the same start: Gauss-point Cauchy stress
    (relative to the largest |sigma| of the FP64 run: the largest over Gauss
    points, its 99.99th percentile, the field's L2 norm and the count of
    points above 1e-3), nodal displacement (relative to the largest |u|), the
    mean axial displacement of the far face x = max (the cantilever's tip),
    the axial reaction on the far face where it is held (the cylinder's
    pushed face), and the largest martensite fraction difference.  The north
    star bounds the stress at 1e-3 and the tip displacement at 1e-4.

    `spread`: plain FP64 runs on the mesh with its coordinates scaled by
    (1 + 2^-24) and (1 - 2^-24), one FP32 ulp, after the same steps -- the
    law's own sensitivity to an FP32-sized change of its input, measured the
    same way (each figure the larger of the two runs').
    The activation test F > F0 and F > Rs (sld_stress_model_160.f90:351,368)
    is discontinuous: a Gauss point whose loading function turns within a
    rounding error of F0 starts transforming one step earlier or later, and
    the stress wave it sends makes neighbours do the same, so after a few
    hundred steps any form whose data carry FP32 rounding parts from FP64 by
    that spread, whatever its arithmetic."""
    g64 = s64.postprocess(gp_sigma=True)["gp_sigma"]
    smax = float(np.abs(g64).max())
    u64 = s64.get("displ")
    X = prob.coord
    far = np.isclose(X[:, 0], X[:, 0].max())
    tip64 = u64[far, 0].mean()
    held = far & (prob.fixno[:, 0] == 1)
    r64 = s64.get("rhsid")[held, 0].sum() if held.any() else None
    n64 = np.linalg.norm(g64)

    def against_fp64(s):
        g = s.postprocess(gp_sigma=True)["gp_sigma"]
        d = np.abs(g - g64).reshape(-1, 6).max(axis=1) / smax
        l2 = float(np.linalg.norm(g - g64) / n64)
        del g
        u = s.get("displ")
        e = {"stress_rel": float(d.max()), "stress_rel_q9999": float(np.quantile(d, 0.9999)),
             "stress_rel_l2": l2, "gauss_points_above_1e-3": int((d > 1e-3).sum()),
             "displacement_rel": float(np.abs(u - u64).max() / np.abs(u64).max()),
             "far_face_ux_rel": float(abs(u[far, 0].mean() - tip64) / max(abs(tip64), 1e-300)),
             "xS_max_abs": float(np.abs(s.state[:, 1, :, 0] - s64.state[:, 1, :, 0]).max())}
        if r64 is not None:
            r = s.get("rhsid")[held, 0].sum()
            e["far_face_reaction_rel"] = float(abs(r - r64) / max(abs(r64), 1e-300))
        return e

    out = {"steps": int(nsteps), "gauss_points": int(g64.size // 6), "max_abs_stress_mpa": smax,
           **against_fp64(s32),
           "bounds": {"stress_rel": 1e-3, "tip_displacement_rel": 1e-4},
           "what": "FP32 form vs plain FP64 form after the same steps from the same start: Gauss-point "
                   "Cauchy stress, nodal displacement, far-face axial displacement, martensite fraction"}
    if spread:
        runs = [against_fp64(s) for s in spread]
        out["law_spread_fp32_ulp"] = {**{k: max(r[k] for r in runs) for k in runs[0]},
                                      "what": "plain FP64 form, mesh coordinates scaled by 1 +- 2^-24, same "
                                              "steps, the larger of the two: the law's own sensitivity at "
                                              "FP32 rounding"}
    return out


def surrogate_leg(args, prob, u0, s64, v64, v32, wsteps, device, spread=None):
    """The FP32 form with the learned surrogate in its element loop: trained
    here by the library's kernels on plain-law paths of the workload's
    materials, switched on after the same warm-up steps of the plain law
    from the same start, the same K steps timed; the plain FP64 run (s64,
    after the same steps) judges its error."""
    import torch
    import alya_sma_b200 as sma
    from alya_sma_b200 import surrogate as S
    net, info = S.train_for(prob, nsamples=args.surrogate_samples, epochs=args.surrogate_epochs, device=device)
    g = sma.ExplicitSolid(prob, precision="fp32", scatter=args.scatter, device=device)
    g.set("displ", u0)
    g.step(wsteps)
    # one element loop judged by the plain FP64 law at the same state and
    # displacement (the FP64 run's after the warm-up steps, loaded into an
    # FP32 context), with the network and with its output held at zero (the
    # method without the learned part)
    j64 = sma.ExplicitSolid(prob, precision="fp64", scatter=args.scatter, device=device)
    j64.set("displ", u0)
    j64.step(wsteps)
    uj, sj = j64.get("displ"), j64.state
    f64 = j64.assemble(uj)["finte"]
    j64.close()
    fscale = float(np.abs(f64).max())
    judged = {"what": "nodal internal forces of one surrogate element loop vs the plain FP64 law's at the same "
                      "state and displacement (the FP64 run's after the warm-up steps), relative to the largest; "
                      "zero_residual: the same loop with the network's output held at zero (the analytic part "
                      "alone)"}
    gj = sma.ExplicitSolid(prob, precision="fp32", scatter=args.scatter, device=device)
    gj.state = sj
    gj.set("displ", uj)
    for name, n in (("zero_residual", S.ZeroResidual(net)), ("network", net)):
        gj.set_surrogate(n, gate=args.surrogate_gate, xs_tol=1e-3, period=SUR_PERIOD)
        d = np.abs(gj.assemble(uj)["finte"] - f64).max(axis=1) / fscale
        judged[name] = {"force_rel_max": float(d.max()), "force_rel_q9999": float(np.quantile(d, 0.9999)),
                        "force_rel_median": float(np.median(d))}
    gj.set_surrogate(net, enable=False)
    d = np.abs(gj.assemble(uj)["finte"] - f64).max(axis=1) / fscale
    judged["fp32_plain_law"] = {"force_rel_max": float(d.max()), "force_rel_q9999": float(np.quantile(d, 0.9999)),
                                "force_rel_median": float(np.median(d))}
    gj.close()
    del f64, sj
    g.set_surrogate(net, gate=args.surrogate_gate, xs_tol=1e-3, period=SUR_PERIOD)
    g.counters(reset=True)
    st = torch.cuda.ExternalStream(g.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    g.step(args.steps)
    b.record(st)
    b.synchronize()
    ngp = prob.nelem * 8
    ms = a.elapsed_time(b)
    v = ngp * args.steps / (ms / 1e3)
    c = g.counters()
    out = {"value": v, "unit": "GP-updates/s", "ms_per_step": ms / args.steps,
           "speedup_vs_plain_fp64": round(v / v64, 3), "speedup_vs_fp32_form": round(v / v32, 3),
           "fallback_fraction": c["sur_fallback"] / (ngp * args.steps),
           "network_evaluations_per_step": ngp // SUR_PERIOD,
           "network_refusal_fraction": c["sur_ood"] * SUR_PERIOD / (ngp * args.steps),
           "return_map_fraction": c["nr_active"] / (ngp * args.steps),
           "tensor_core_status": g.surrogate_status(), "gate": args.surrogate_gate,
           "network": "14 -> 64x4 (SiLU) -> 13, BF16 tcgen05.mma with FP32 accumulation in TMEM",
           "training": info, "judged_by_plain_law": judged,
           "error_vs_fp64": compare_forms(prob, g, s64, wsteps + args.steps, spread)}
    g.close()
    return out


def cpu_baseline(prob, u0, budget_s=15.0, max_steps=50):
    """The oracle's central-difference step (colour-parallel element loop,
    OpenMP over all host threads, compiled with -march=native on this host)
    on the full mesh, as many steps as fit in about budget_s seconds."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    o = O.Problem(prob, nthreads=threads, native=True)
    o.displ[:] = u0
    o.run(prob.dtime, 1)                      # warm-up (page-in, thread pool)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.run(prob.dtime, 1)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": prob.nelem * 8 * steps / dt, "unit": "GP-updates/s", "cores": threads,
            "kind": "port", "sample": f"{steps} central-difference steps of the full "
                                      f"{prob.nelem}-element mesh ({dt:.1f} s), "
                                      + ("-O3 -march=native" if o.native else "-O3 -march=x86-64-v3")
                                      + f" -fopenmp on {cpu_model()}"}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def run_reference(args):
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return 0
    from alya_sma_b200 import problem as P
    if args.partition is None:
        args.partition = world > 1 and args.workload != "ensemble"
    prob = build_problem(args.workload, args.div, layers=args.layers)
    sharded = args.workload == "ensemble" and world > 1
    gp_all = prob.nelem * 8 * (1 if (sharded or args.partition) else world)
    u0 = P.prestrain(prob, args.prestrain)
    base = cpu_baseline(prob, u0, budget_s=15.0, max_steps=max(2, args.steps))
    line = {"impl": "reference", "metric": "Gauss-point updates/s (explicit SMA step)",
            "value": base["value"], "unit": "GP-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": prob.nelem * 8 / base["value"] * 1e3, "higher_is_better": True,
            "scaling": "strong" if (args.workload == "ensemble" and world > 1) else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": arm_config(args, world, prob.nelem, prob.npoin, gp_all, working_set(prob, args.precision)),
            "reference_path": "the oracle's FP64 restatement of the reference CPU step (the Fortran reference "
                              "does not build here), OpenMP colour-parallel on the host cores",
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "GP-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_partitioned(args, rank, world, local):
    """--partition: every rank builds the whole mesh, keeps its element slab
    and steps it with the others: interface elements, the shared rows sent
    to and received from the neighbouring slabs (NCCL send/recv under
    torchrun) while the interior elements compute, the sums written back,
    the nodal update.  value = the mesh's Gauss points (each counted once)
    x K / the slowest rank's time.  The per-step events of a second window
    time the part's element launch, the (unoverlapped) exchange and the
    nodal launch."""
    import torch
    import alya_sma_b200 as sma
    from alya_sma_b200 import dist as D
    from alya_sma_b200 import partition as PT
    from alya_sma_b200 import problem as P
    if args.precision == "surrogate":
        raise SystemExit("--partition runs the fp32 or fp64 form")
    prob = build_problem(args.workload, args.div, layers=args.layers)
    group = torch.distributed.group.WORLD if world > 1 else None
    ps = PT.PartitionedSolid(prob, nparts=1, precision=args.precision, scatter=args.scatter, device=local,
                             group=group, block=args.block)
    part = ps.solids[rank if group is not None else 0]
    ps.set("displ", P.prestrain(prob, args.prestrain))
    ps.step(max(3, args.warmup))
    stream = torch.cuda.ExternalStream(part.stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    clocks = Clocks(local)
    barrier()
    clocks.start()
    l0 = part.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ps.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ck = clocks.stop()
    launches = part.kernel_launches - l0
    ms = D.max_over_ranks(e0.elapsed_time(e1), "cuda")
    ngp = prob.nelem * 8
    value = ngp * args.steps / (ms / 1e3)

    # per-phase times of this rank's part over a second window
    L = sma.lib()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    sma._check(L.sma_step_prologue(part._ctx))
    for n in range(args.steps):
        ev[n][0].record(stream)
        sma._check(L.sma_step_elements(part._ctx))
        ev[n][1].record(stream)
        ps._exchange()
        ev[n][2].record(stream)
        sma._check(L.sma_step_nodes(part._ctx, int(n == args.steps - 1)))
        ev[n][3].record(stream)
    torch.cuda.synchronize()
    el_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / args.steps
    ex_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / args.steps
    nd_ms = sum(e[2].elapsed_time(e[3]) for e in ev) / args.steps
    k = rank if group is not None else 0
    q, _ = PT.sub_problem(prob, ps.parts[k], np.ones(prob.npoin, bool))
    # e2e: every rank's element-loop C-ABI call on its slab with pinned host
    # buffers (its displacement in, its residual out), the job's Gauss points
    # over the slowest rank's time
    npart = part.npoin
    hd = torch.zeros((npart, 3), dtype=torch.float64).pin_memory()
    hr = torch.zeros((npart, 3), dtype=torch.float64).pin_memory()
    hd.copy_(torch.from_numpy(part.get("displ")))
    dnp, rnp = hd.numpy(), hr.numpy()
    for _ in range(3):
        sma._check(L.sma_assemble(part._ctx, dnp.ctypes.data, 0.0, rnp.ctypes.data, None, None, None, None))
        part.end_step()
    ke = max(10, args.steps // 20)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        sma._check(L.sma_assemble(part._ctx, dnp.ctypes.data, 0.0, rnp.ctypes.data, None, None, None, None))
        part.end_step()
    te = D.max_over_ranks(time.perf_counter() - t0, "cuda")
    e2e = {"value": ngp * ke / te, "unit": "GP-updates/s", "h2d_bytes_per_step": 3 * npart * 8,
           "d2h_bytes_per_step": 3 * npart * 8,
           "boundary": "sma_assemble on each rank's slab (host displ in, host rhsid out), slowest rank's time"}
    alg = algorithmic_bytes(q, args.precision)
    peak, peak_kind = measured_peaks()
    achieved = alg / (el_ms / 1e3) / 1e9
    prof = load_profile(args.precision, args.workload, q.nelem) if (world == 1 and args.div == 1
                                                                       and not args.layers) else None
    roofline = {"bound": "hbm", "kernel": "k_element", "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": prof["traffic"] if prof else None, "algorithmic_bytes_per_launch": alg,
                "launch_ms": round(el_ms, 4), "exchange_ms": round(ex_ms, 4), "nodal_launch_ms": round(nd_ms, 4),
                "window": "rank 0's part, per-step CUDA events on its stream over a second K-step window",
                "note": "compute-bound kernel: the FP32/FP64 pipes, not HBM, bind it"}
    if rank == 0:
        line = {"metric": "Gauss-point updates/s (explicit SMA step)", "value": value,
                "unit": "GP-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32+f64" if args.precision == "fp32" else "f64",
                "data": "synthetic",
                "config": arm_config(args, world, prob.nelem, prob.npoin, ngp, working_set(prob, args.precision)),
                "launch": {"scatter": args.scatter, **part.launch_info(), "dtime": prob.dtime,
                           "shared_nodes": ps.nshared},
                "roofline": roofline, "gpu_launches": launches, "clocks": ck, "e2e": e2e}
        print(json.dumps(line))
    ps.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.write_profile:
        prob = build_problem(args.workload, args.div, layers=args.layers)
        note = (f"captured on the {prob.nelem}-element case (--layers {args.layers}); bench.py scales "
                "traffic and instructions to the bench mesh by element count") if args.layers else ""
        write_profile(args.write_profile, args.precision, args.workload, prob.nelem, note)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import alya_sma_b200 as sma
    rank, world, local = dist_env()
    torch.cuda.set_device(local)                              # before NCCL binds the rank's device
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    if args.partition is None:
        args.partition = world > 1 and args.workload != "ensemble"
    if args.partition:
        return run_partitioned(args, rank, world, local)
    prob = build_problem(args.workload, args.div, rank, world, layers=args.layers)
    nelem, ngp = prob.nelem, prob.nelem * 8
    sharded = args.workload == "ensemble" and world > 1       # strong scaling: fixed total work

    from alya_sma_b200 import problem as P
    u0 = P.prestrain(prob, args.prestrain)
    block, scatter, tuned, plan = args.block, args.scatter, None, None
    variant = "auto"
    if args.autotune and args.workload == "ensemble":
        # per specimen-size bucket: each bucket's element range its own block
        from alya_sma_b200 import tune
        tuned = tune.tune_buckets(prob, precision="fp32" if args.precision == "surrogate" else args.precision,
                                  displ=u0, device=local)
        plan = tuned["plan"]
    elif args.autotune:
        from alya_sma_b200 import tune
        tuned = tune.tune(prob, precision=args.precision, displ=u0, steps=10, warmup=3, device=local)
        block, scatter, variant = tuned["block"], tuned["scatter"], tuned["variant"]
    args.scatter = scatter
    # --precision surrogate: the FP32 form with the learned surrogate in its
    # element loop is the timed form (trained first; the warm-up runs the
    # plain law, as the surrogate leg of the default run does)
    net, sur_info = None, None
    prec = "fp32" if args.precision == "surrogate" else args.precision
    if args.precision == "surrogate":
        from alya_sma_b200 import surrogate as S
        net, sur_info = S.train_for(prob, nsamples=args.surrogate_samples, epochs=args.surrogate_epochs,
                                    device=local)
    solid = sma.ExplicitSolid(prob, precision=prec, scatter=scatter, block=block,
                              device=local, variant=variant)
    if plan:
        solid.set_launch_plan([e for _, e, _ in plan], [blk for _, _, blk in plan])
    launch_info = solid.launch_info()
    solid.set("displ", u0)
    stream = torch.cuda.ExternalStream(solid.stream)
    solid.step(max(3, args.warmup))
    if net is not None:
        solid.set_surrogate(net, gate=args.surrogate_gate, xs_tol=1e-3, period=SUR_PERIOD)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # the state at the start of the timed region, to replay the same window
    # with per-launch events (the element work depends on how many Gauss
    # points transform, so a different window would time different work)
    import tempfile
    ckpt = os.path.join(tempfile.mkdtemp(prefix="sma_bench_"), f"window_r{rank}.bin")
    solid.save(ckpt)

    solid.counters(reset=True)                 # the window's physics, counted by the kernels

    # ---- timed region: K device-resident steps (CUDA graphs) ---------------
    clocks = Clocks(local)
    barrier()
    clocks.start()
    l0 = solid.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solid.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ck = clocks.stop()
    launches = solid.kernel_launches - l0
    ms = e0.elapsed_time(e1)
    cnt = solid.counters()
    physics = {"gauss_points_in_return_map_per_step": round(cnt["nr_active"] / args.steps),
               "return_map_failures": cnt["nr_failed"], "det_F_nonpositive": cnt["neg_det"],
               "nonfinite": cnt["nonfinite"]}
    if net is not None:
        physics["surrogate_fallback_fraction"] = cnt["sur_fallback"] / (ngp * args.steps)
        physics["surrogate_network_refusal_fraction"] = cnt["sur_ood"] * SUR_PERIOD / (ngp * args.steps)
        physics["surrogate_training"] = sur_info
    ngp_all = world * ngp                                      # replicas: the same mesh per rank
    nelem_all, npoin_all, wset_all = nelem, prob.npoin, working_set(prob, args.precision)
    from alya_sma_b200 import dist as D                       # (identity on one rank)
    if world > 1:
        ms = D.max_over_ranks(ms, "cuda")                      # the slowest rank sets the time
        if sharded:
            ngp_all = int(D.sum_over_ranks(ngp, "cuda"))       # each specimen counted once
            nelem_all = int(D.sum_over_ranks(nelem, "cuda"))
            npoin_all = int(D.sum_over_ranks(prob.npoin, "cuda"))
            wset_all = float(D.sum_over_ranks(wset_all, "cuda"))
    value = ngp_all * args.steps / (ms / 1e3)

    # ---- per-kernel device times (roofline of the element kernel): the same
    # K steps replayed from the checkpoint, CUDA events around every launch
    # on the library's stream ------------------------------------------------
    solid.load(ckpt)
    os.remove(ckpt)
    os.rmdir(os.path.dirname(ckpt))
    if net is not None:                        # eps_tr derived again from the window's start
        solid.set_surrogate(net, gate=args.surrogate_gate, xs_tol=1e-3, period=SUR_PERIOD)
    solid.set_timing(True)
    solid.step(args.steps)
    tm = solid.timers()
    solid.set_timing(False)
    el_ms = tm["element"][0] / max(1, tm["element"][1])
    nd_ms = tm["nodal"][0] / max(1, tm["nodal"][1])
    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes(prob, args.precision)
    achieved = alg / (el_ms / 1e3) / 1e9
    prof = load_profile(args.precision, args.workload, nelem) if (args.div == 1 and not args.layers) else None
    roofline = {"bound": "hbm", "kernel": "k_element", "achieved": round(achieved, 1),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": prof["traffic"] if prof else None,
                "algorithmic_bytes_per_launch": alg,
                "algorithmic_bytes_per_gauss_point": round(alg / ngp, 1),
                "launch_ms": round(el_ms, 4), "nodal_launch_ms": round(nd_ms, 4),
                "window": "the K timed steps replayed from a checkpoint of their start, "
                          "CUDA events around each launch on the library stream",
                "profile": (f"profiles/k_element_{args.precision}_{args.workload}.json, scaled from "
                            f"{prof['scaled_from_elements']} elements" if prof else
                            "no ncu summary of this kernel build and workload: traffic not reported"),
                "note": "compute-bound kernel: the FP32/FP64 pipes, not HBM, bind it"}
    if prof and prof["warp_inst"]:
        # instruction-issue roofline: warp instructions per launch (ncu) over
        # the measured launch time, against 4 issue slots per SM per clock
        rate = prof["warp_inst"] / (el_ms / 1e3)
        peak_i = 4 * prof["sms"] * ((ck or {}).get("sm_mhz") or 1965.0) * 1e6
        roofline["issue"] = {"warp_inst_per_launch": round(prof["warp_inst"]),
                             "achieved_ginst_s": round(rate / 1e9, 1),
                             "peak_ginst_s": round(peak_i / 1e9, 1),
                             "frac": round(rate / peak_i, 4)}

    extras = {}
    if not args.no_extras and rank == 0 and args.precision == "fp32":
        # the plain FP64 form: the same steps from the same start, its K
        # steps timed like the FP32 window; then both forms compared
        wsteps = max(3, args.warmup)
        s64 = sma.ExplicitSolid(prob, precision="fp64", scatter=args.scatter, device=local)
        s64.set("displ", u0)
        s64.step(wsteps)
        st64 = torch.cuda.ExternalStream(s64.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st64)
        s64.step(args.steps)
        b.record(st64)
        b.synchronize()
        v64 = ngp * args.steps / (a.elapsed_time(b) / 1e3)
        extras["plain_fp64"] = {"value": v64, "unit": "GP-updates/s", "steps": args.steps,
                                "ms_per_step": a.elapsed_time(b) / args.steps}
        extras["speedup_vs_plain_fp64"] = round(value / world / v64, 3)
        # the law's own spread: FP64 on the mesh moved by one FP32 ulp
        import copy
        spread = []
        for sign in (1.0, -1.0):
            pu = copy.copy(prob)
            pu.coord = prob.coord * (1.0 + sign * 2.0 ** -24)
            su = sma.ExplicitSolid(pu, precision="fp64", scatter=args.scatter, device=local)
            su.set("displ", u0)
            su.step(wsteps + args.steps)
            spread.append(su)
        extras["error_vs_fp64"] = compare_forms(prob, solid, s64, wsteps + args.steps, spread)
        if args.surrogate:
            extras["surrogate"] = surrogate_leg(args, prob, u0, s64, v64, value / world, wsteps, local, spread)
        for su in spread:
            su.close()
        s64.close()
    if not args.no_extras:
        # e2e on every rank: the element-loop C-ABI call with pinned host
        # buffers, host copies inside the timed region; the job's Gauss points
        # over the slowest rank's time
        npoin = prob.npoin
        hd = torch.zeros((npoin, 3), dtype=torch.float64).pin_memory()
        hr = torch.zeros((npoin, 3), dtype=torch.float64).pin_memory()
        hd.copy_(torch.from_numpy(solid.get("displ")))
        dnp, rnp = hd.numpy(), hr.numpy()
        L = sma.lib()
        ctx = solid._ctx
        for _ in range(3):
            sma._check(L.sma_assemble(ctx, dnp.ctypes.data, 0.0, rnp.ctypes.data, None, None, None, None))
            solid.end_step()
        ke = max(10, args.steps // 20)
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            sma._check(L.sma_assemble(ctx, dnp.ctypes.data, 0.0, rnp.ctypes.data, None, None, None, None))
            solid.end_step()
        te = D.max_over_ranks(time.perf_counter() - t0, "cuda")
        # the host link alone: the same bytes copied from and to the same
        # pinned buffers, both directions at once on two streams, the same
        # number of times -- the floor the call's copies set
        dd = torch.empty((npoin, 3), dtype=torch.float64, device=local)
        dr = torch.empty((npoin, 3), dtype=torch.float64, device=local)
        s_in, s_out = torch.cuda.Stream(local), torch.cuda.Stream(local)
        for rep in range(2):                                  # one untimed round, one timed
            barrier()
            t1 = time.perf_counter()
            for _ in range(ke):
                with torch.cuda.stream(s_in):
                    dd.copy_(hd, non_blocking=True)
                with torch.cuda.stream(s_out):
                    hr.copy_(dr, non_blocking=True)
                s_in.synchronize()
                s_out.synchronize()
            tl = time.perf_counter() - t1
        tl = D.max_over_ranks(tl, "cuda")
        del dd, dr
        extras["e2e"] = {"value": ngp_all * ke / te, "unit": "GP-updates/s",
                         "h2d_bytes_per_step": 3 * npoin * 8, "d2h_bytes_per_step": 3 * npoin * 8,
                         "boundary": "sma_assemble (element loop, host displ in, host rhsid out)",
                         "ms_per_step": round(te / ke * 1e3, 4),
                         "host_link": {"copies_ms_per_step": round(tl / ke * 1e3, 4),
                                       "gb_s_each_way": round(3 * npoin * 8 / (tl / ke) / 1e9, 1),
                                       "frac": round(tl / te, 3),
                                       "what": "pinned copies of the same bytes, both directions at once, "
                                               "no kernels: the floor of the call's time"}}
        # the step boundary (sma_explicit_step): the state stays on the
        # device; the host asks for K steps and reads back, as the step's
        # result, the axial displacement history of the far face's first node
        # (the witness rows, one per step); wall time around the calls
        far = int(np.flatnonzero(np.isclose(prob.coord[:, 0], prob.coord[:, 0].max()))[0])
        solid.set_witness([3 * far], args.steps)
        solid.step(2)
        solid.witness()
        solid.set_witness([3 * far], args.steps)
        barrier()
        t0 = time.perf_counter()
        solid.step(args.steps)
        hist = solid.witness()
        ts = D.max_over_ranks(time.perf_counter() - t0, "cuda")
        assert hist.shape[0] == args.steps and np.isfinite(hist).all()
        extras["e2e_step_boundary"] = {"value": ngp_all * args.steps / ts, "unit": "GP-updates/s",
                                       "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8,
                                       "ms_per_step": round(ts / args.steps * 1e3, 4),
                                       "boundary": "sma_explicit_step over the K steps (state resident), the "
                                                   "far-face displacement history read back"}
        if world == 1:
            extras["cpu_baseline"] = cpu_baseline(prob, u0)
    if world > 1:
        torch.distributed.barrier()

    if rank == 0:
        line = {"metric": "Gauss-point updates/s (explicit SMA step)", "value": value,
                "unit": "GP-updates/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if sharded else "weak", "vs_baseline": None,
                "dtype": {"fp32": "f32+f64", "fp64": "f64", "surrogate": "bf16+f32+f64"}[args.precision],
                "data": "synthetic",
                "config": arm_config(args, world, nelem_all, npoin_all, ngp_all, wset_all),
                "launch": {"scatter": args.scatter, **launch_info, "autotuned": bool(tuned), "dtime": prob.dtime,
                           "launch_plan": ([{"bucket_elements": bk, "end": e, "block": blk} for bk, e, blk in plan]
                                           if plan else None),
                           **({"autotune_step_ms": {"plan": round(tuned["step_ms"], 4),
                                                    "single_default_launch": round(tuned["default_step_ms"], 4)}}
                              if tuned and "default_step_ms" in tuned else {})},
                "roofline": roofline, "gpu_launches": launches, "clocks": ck, "physics": physics}
        line.update(extras)
        print(json.dumps(line))
    solid.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
