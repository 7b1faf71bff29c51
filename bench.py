"""Benchmark: Darcy solve seconds to relative residual 1e-10 on the 1e6-cell annulus.

Workload (one step = one solve from zero initial guess): annulus 0.3 < r < 1 with exact circular
arcs, 1e6 seeded Voronoi + 20 Lloyd cells, k = 0, lognormal K (exponential covariance, sigma 2,
correlation length 0.1), pressure 1 on r = 0.3 and 0 on r = 1, FP32 local operators and inner
MINRES under FP64 iterative refinement (the headline), the plain FP64 MINRES solve timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--cells C]

Multi-GPU: replicas only (the reference solver does not partition; every configuration fits one
GPU); each rank solves its own seeded problem, no data-path collective; value = max over ranks.
``--impl reference`` times the reference CPU algorithm restated in the oracle (element matrices,
CSR assembly, GMRES(100) + ILU(0), rtol 1e-10) on rank 0 over a bounded sample.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "wsl-code_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "Darcy solve s @1e-10 vs FP64 oracle: FP32-refined vs FP64 GPU; HBM GB/s; grad/solve"
CACHE = os.path.join(ROOT, "wsl-code_b200", "_meshcache")
INNER_TOL = 1e-6  # FP32 inner MINRES: relative reduction per refinement step
PARITY_TOL = 1e-12  # residual of the solves compared with the oracle
FD_TOL = 1e-14  # residual of the FP64 forward solves of the finite-difference checks (the FP64 floor)
GRAD_TOL = 1e-12  # residual of the FP64 adjoint solve of the gradient checks
CORR_TOL = 1e-12  # residual, relative to its right-hand side, of the FP64 correction solves of the FD check


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--cpu-sample-cells", type=int, default=8000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle-checks", action="store_true", help="skip the oracle's LU checks of C2 and C4")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--profile", action="store_true", help="short fixed run for profilers (applies + 2 solves)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the gradient workload")
    ap.add_argument("--adjoint-cells", type=int, default=250000)
    ap.add_argument("--fd-directions", type=int, default=20)
    ap.add_argument("--no-assembled", action="store_true", help="skip the assembled cuSPARSE comparator")
    ap.add_argument("--no-config1", action="store_true", help="skip the 250k-cell disk k=0/k=1 leg")
    ap.add_argument("--config1-cells", type=int, default=250000)
    ap.add_argument("--no-ms", action="store_true", help="skip the Maxwell-Stefan leg")
    ap.add_argument("--ms-steps", type=int, default=100)
    ap.add_argument("--eager", action="store_true", help="with --profile: host-driven Krylov batches, no graph")
    ap.add_argument("--profile-ms", action="store_true", help="with --profile: also Maxwell-Stefan applies and steps")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_bytes(kernel, cells):
    """DRAM bytes (read + write) of one launch of `kernel` from the committed ncu summary
    profiles/traffic.json, scaled by cells when it was captured on another mesh size."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)[kernel]
        return t["bytes"] * cells / t["cells"]
    except Exception:
        return None


def disk_mesh(cells, seed):
    """Voronoi + Lloyd mesh of the unit disk with exact arcs (cached on disk)."""
    import numpy as np
    from vemgpu import meshgen
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"disk_{cells}_s{seed}.npz")
    if os.path.exists(path):
        z = np.load(path)
        return {k: z[k] for k in z.files}
    mesh = meshgen.voronoi_mesh(cells, "disk", seed=seed)
    mesh = {k: v for k, v in mesh.items() if isinstance(v, np.ndarray)}
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, **mesh)
    os.replace(tmp, path)
    return mesh


def annulus_problem(cells, seed):
    """Mesh (cached on disk) and log-permeability field of the workload."""
    import numpy as np
    from vemgpu import fields, meshgen
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"annulus_{cells}_s{seed}.npz")
    if os.path.exists(path):
        z = np.load(path)
        mesh = {k: z[k] for k in z.files}
    else:
        mesh = meshgen.voronoi_mesh(cells, "annulus", seed=seed)
        mesh = {k: v for k, v in mesh.items() if isinstance(v, np.ndarray)}
        tmp = path + f".{os.getpid()}.tmp.npz"
        np.savez(tmp, **mesh)
        os.replace(tmp, path)
    theta = fields.gaussian_field(fields.cell_centroids(mesh), sigma=2.0, corr=0.1, seed=seed + 1)
    return mesh, theta


def apply_bytes(g, mesh, fp):
    """Algorithmic bytes of one apply (k = 0): packed A_E + int32 map + cell id per cell, x read
    once and y written once (no multiplier, no W at k = 0)."""
    import numpy as np
    s = 4 if fp == 32 else 8
    ne = np.diff(mesh["cell_ptr"]).astype(np.int64)
    per_cell = s * ne * (ne + 1) // 2 + 4 * ne + 4
    return int(per_cell.sum() + s * 2 * g.N)


class ClockSampler:
    def __init__(self, path):
        self.path, self.p = path, None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()
            self.f.close()

    def summary(self, device):
        import statistics
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    t = [c.strip() for c in line.split(",")]
                    if len(t) >= 9 and t[0] == str(device):
                        rows.append(t)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def cpu_info():
    """Host CPU model and logical core count (the CPU legs run on this host)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count() or 1}


def _load_by_path(name, path):
    """A module loaded from its file alone (no package __init__, so no library is mapped)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_sample(args):
    """Mesh and log permeability of the CPU reference runs: the oracle's own scipy Voronoi + Lloyd
    annulus (oracle/meshgen_ref.py) and the same Gaussian random field generator as the GPU
    workload (sigma 2, correlation length 0.1), for the bounded sample size."""
    import meshgen_ref
    fields = _load_by_path("vg_fields", os.path.join(ROOT, "wsl-code_b200", "vemgpu", "fields.py"))
    mesh = meshgen_ref.voronoi_mesh(args.cpu_sample_cells, "annulus", seed=args.seed)
    theta = fields.gaussian_field(fields.cell_centroids(mesh), sigma=2.0, corr=0.1, seed=args.seed + 1)
    return mesh, theta


def cpu_solve(mesh, theta, threads, problem=None):
    """The reference CPU algorithm restated in the oracle: element matrices, CSR assembly (OpenMP
    over `threads` cores) and GMRES(100) + ILU(0) to rtol 1e-10 (one core, like PETSc on
    PETSC_COMM_SELF). Returns (x, iterations, times)."""
    import oracle as O
    return O.reference_solve(mesh, k=0, nq=9, ng=9, geom=O.GEOM_ARCS, problem=problem or O.PROB_ANNULUS,
                             bc=O.BC_PRESSURE, theta=theta, threads=threads, rtol=1e-10, maxit=2000000)


# The same CPU path run once on the whole 1M-cell workload (the bench's mesh and permeability, seed
# 2026; assembly on 16 threads, GMRES(100)+ILU(0) on one) on a 16-core Intel Xeon build host, not
# on the GPU box: too long for the arm's time limit, so it is reported beside the measured sample.
FULL_CPU_1M = {"value": 7257.8, "unit": "s", "assembly_s": 17.2, "gmres_ilu_s": 7231.5, "iterations": 6425,
               "true_relative_residual": 9.94e-11, "kind": "measured once on the build host, not in this run"}


def reference_arm(args, rank):
    """The reference's CPU path for this workload, measured: every step is one full CPU solve
    (assembly + GMRES(100)+ILU(0), rtol 1e-10) of a bounded sample of the workload, the
    annulus family at --cpu-sample-cells cells. `value` is the measured seconds per sample solve
    on the sample's own cell count; the 1M-cell workload itself takes hours on one core and is
    not run (a linear lower-bound estimate is reported beside the value, labelled as such)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    mesh, theta = reference_sample(args)
    cells = len(mesh["cell_ptr"]) - 1
    times, asm, sol = [], [], []
    for i in range(args.warmup + args.steps):
        _, it, tm = cpu_solve(mesh, theta, threads)
        if i >= args.warmup:
            times.append(tm["assembly_s"] + tm["solve_s"])
            asm.append(tm["assembly_s"])
            sol.append(tm["solve_s"])
    value = sum(times) / len(times)
    cpu = cpu_info()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"annulus 0.3<r<1, {cells} Voronoi+Lloyd cells (exact arcs), k=0, lognormal K "
                                   f"(sigma 2, corr 0.1), p=1 inner / 0 outer, to ||b-Ax||/||b|| <= 1e-10: a bounded "
                                   f"sample of the {args.cells}-cell workload",
                       "cells": cells, "sample_of_cells": args.cells, "k": 0, "nq": 9, "ng": 9,
                       "parallelism": "CPU: assembly on all cores, GMRES+ILU(0) on one"},
            "cpu": cpu, "assembly_s": sum(asm) / len(asm), "gmres_ilu_s": sum(sol) / len(sol), "iterations": it,
            "estimate_full_workload_s": {"value": value * args.cells / cells, "kind": "estimate, not measured: "
                                         "linear in cells, a lower bound (GMRES+ILU iterations grow with the mesh)"},
            "full_workload_measured_once": FULL_CPU_1M if args.cells == 1000000 else None,
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port",
                             "sample": f"reference algorithm restated (oracle): element matrices + CSR assembly "
                                       f"({threads} threads) + GMRES(100)+ILU(0) rtol 1e-10 (1 thread) on a {cells}-cell "
                                       f"annulus of the same family (oracle mesh generator), measured per solve, "
                                       f"{it} iterations; CPU {cpu['model']}"},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _oracle_worker(kind, mesh_path, theta, conn):
    """Spawned child process: the oracle's CPU FP64 checks on the 250k-cell meshes (numpy, scipy
    and the oracle library only; no CUDA). Runs beside the GPU legs; talks through `conn`.

    kind "c2": the disk problem (p = sin(pi x) sin(pi y), K = I, Dirichlet pressure), k = 0 by
    sparse LU (the golden discrete solution) with its six error figures; then, for the k = 1 GPU
    solution it receives, the oracle's own residual ||b - K x|| / ||b|| and error figures (a sparse
    LU of the 3M-unknown k = 1 system exceeds SuperLU's limits here).
    kind "c4": the annulus with log permeability theta: one sparse LU gives the forward solution;
    for the observation rows and data it receives, J, dJ/dx, the adjoint lam = K^-T dJ/dx and the
    per-cell gradient lam_E^T A_E x_E (the CPU FP64 gradient)."""
    import numpy as np
    import scipy.sparse.linalg as spla
    import oracle as O
    try:
        z = np.load(mesh_path)
        mesh = {k: z[k] for k in z.files}
        t0 = time.time()
        if kind == "c2":
            o = O.Oracle(mesh, k=0, nq=9, ng=9, geom=O.GEOM_ARCS, problem=O.PROB_SINSIN, bc=O.BC_PRESSURE, threads=4)
            xo, _, _ = o.solve_direct()
            conn.send({"x": xo, "seconds": time.time() - t0, "errors": o.errors(xo), "N": o.N})
            del o
            x1 = conn.recv()
            if x1 is not None:
                o1 = O.Oracle(mesh, k=1, nq=9, ng=9, geom=O.GEOM_ARCS, problem=O.PROB_SINSIN, bc=O.BC_PRESSURE,
                              threads=4)
                K1, b1 = o1.system()
                r = float(np.linalg.norm(b1 - K1 @ x1) / np.linalg.norm(b1))
                conn.send({"residual": r, "errors": o1.errors(x1), "N": o1.N})
        else:
            o = O.Oracle(mesh, k=0, nq=9, ng=9, geom=O.GEOM_ARCS, problem=O.PROB_ANNULUS, bc=O.BC_PRESSURE,
                         theta=theta, threads=4)
            K, b = o.system()
            lu = spla.splu(K.tocsc(), permc_spec="COLAMD")
            x = lu.solve(b)
            t_lu = time.time() - t0
            req = conn.recv()
            if req is not None:
                idx, data = req
                r = x[idx] - data
                dJdx = np.zeros(o.N)
                np.add.at(dJdx, idx, 2.0 * r)
                lam = lu.solve(dJdx, trans="T")
                g = o.adjoint_contract(x, lam)
                conn.send({"J": float(r @ r), "g": g, "x_obs": x[idx], "seconds": t_lu, "N": o.N})
    except Exception as e:  # reported by the parent, never silently dropped
        conn.send({"error": f"{type(e).__name__}: {e}"})
    finally:
        conn.close()


class OracleJob:
    """One spawned oracle check (spawn context: no state of the parent's CUDA context)."""

    def __init__(self, kind, mesh_path, theta=None):
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        self.conn, child = ctx.Pipe()
        self.p = ctx.Process(target=_oracle_worker, args=(kind, mesh_path, theta, child), daemon=True)
        self.p.start()
        child.close()

    def send(self, obj):
        self.conn.send(obj)

    def recv(self, timeout=1800):
        if not self.conn.poll(timeout):
            raise RuntimeError("oracle check did not answer in time")
        out = self.conn.recv()
        if isinstance(out, dict) and "error" in out:
            raise RuntimeError("oracle check failed: " + out["error"])
        return out

    def close(self):
        try:
            self.conn.close()
        finally:
            self.p.join(timeout=60)
            if self.p.is_alive():
                self.p.terminate()


def adjoint_leg(args, rank, job=None):
    """Config C4 (250k-cell annulus, lognormal K): J = sum over 64 seeded interior points of
    (p_h - d)^2, the data d being the pressures of a solve with a second seeded K field. Reports:
    * the adjoint (vg_adjoint_grad: adjoint solve + per-cell contraction) against the forward
      solve, both device-timed, in mixed and FP64 modes (solves to 1e-10);
    * the gradient (forward solve to FD_TOL, adjoint solve to GRAD_TOL) against the oracle's CPU
      FP64 gradient (sparse LU of the forward system, adjoint by the transposed factors, per-cell
      contraction; `job`);
    * FP64 central differences (step 1e-6) of J along 20 seeded unit directions, each J from a
      solve to FD_TOL started from the base solution, against the adjoint's directional derivatives,
      relative to the largest directional derivative; and the same central differences with the
      numerator formed from the pressure corrections x(theta +- step v) - x0 (solved for directly),
      which removes the cancellation between the two values of J."""
    import numpy as np
    import torch
    import vemgpu
    from vemgpu import fields, observe
    cells = args.adjoint_cells
    mesh, _ = annulus_problem(cells, args.seed)
    cen = fields.cell_centroids(mesh)
    th = fields.gaussian_field(cen, sigma=2.0, corr=0.1, seed=args.seed + 11 + rank)
    th_data = fields.gaussian_field(cen, sigma=2.0, corr=0.1, seed=args.seed + 21 + rank)
    h = vemgpu.DarcyGpu(mesh, k=0, nq=9, ng=9, geometry="arcs", problem="annulus", bc="pressure", theta=th_data)
    obs = observe.PointObservation(h, mesh, observe.seeded_points(64, args.seed + 12))
    xd, _ = h.solve(tol=1e-12)
    obs.data = obs.pressure(xd).clone()
    if job is not None:
        job.send((obs.index.cpu().numpy(), obs.data.cpu().numpy()))
    h.set_log_permeability(th)
    out = {"cells": h.nc, "observations": 64, "data": "pressures of a second seeded K field"}
    for mode in ("mixed", "fp64"):
        opts = dict(mode=mode, tol=1e-10, inner_tol=INNER_TOL)
        fw, ad = [], []
        for i in range(4):
            x, info = h.solve(**opts)
            dJdx = torch.autograd.functional.vjp(obs, x)[1]
            g, ainfo = h.adjoint_grad(x, dJdx, **opts)
            if i:
                fw.append(info["seconds"])
                ad.append(ainfo["seconds"])
        torch.cuda.synchronize()
        out[mode] = {"forward_s": float(np.mean(fw)), "adjoint_s": float(np.mean(ad)),
                     "grad_over_solve": float(np.mean(ad) / np.mean(fw)),
                     "forward_iterations": info["iterations"], "adjoint_iterations": ainfo["iterations"]}

    def solve_tight(guess=None):
        x = h.zeros() if guess is None else guess.clone()
        try:
            _, info = h.solve(x=x, mode="fp64", tol=FD_TOL, guess=guess is not None)
            return x, info["residual"]
        except vemgpu.VemGpuError:
            return x, float("nan")  # the FP64 floor was reached before FD_TOL: x is the last iterate
    x0, res0 = solve_tight()
    J = float(obs(x0))
    dJdx = torch.autograd.functional.vjp(obs, x0)[1]
    grad, ginfo = h.adjoint_grad(x0, dJdx, mode="fp64", tol=GRAD_TOL)
    gn = float(torch.linalg.norm(grad))
    out["J"], out["grad_norm"], out["tight_residual"] = J, gn, res0
    if job is not None:
        r = job.recv()
        gc = r["g"]
        gg = grad.cpu().numpy()
        out["cpu_gradient"] = {"max_abs_diff_over_max_abs": float(np.abs(gg - gc).max() / np.abs(gc).max()),
                               "J_rel_diff": abs(J - r["J"]) / abs(r["J"]), "oracle_seconds": r["seconds"],
                               "oracle": "sparse LU of the 1M-unknown system, adjoint by the transposed factors"}
        job.close()

    # Cancellation-free central differences. K(theta) = [M(theta), -W^T; W, 0] with the flux block
    # M(theta) = sum_E exp(-theta_E) M_E, so for theta' = theta + sigma step v
    #   K(theta') x0 = K(theta) x0 + [sum_E s_E exp(-theta_E) M_E u0; 0],  s_E = expm1(-sigma step v_E),
    # u0 the flux part of x0. The perturbation term is formed by one apply of u0 with the log
    # permeability theta - log(s + m) (m a power of two above 2 max|s|: a benign uniform shift of the
    # field) less m times the apply of u0 at theta (exact scaling): its rounding error is relative to
    # m |s| M u0, not to K x0. The correction e = x(theta') - x0 solves
    # K(theta') e = (b - K(theta) x0) - perturbation, an FP64 solve to CORR_TOL relative to its own
    # right-hand side, and J(+) - J(-) = sum_o (p+ - p-)(p+ + p- - 2 d_o) is formed from the two
    # corrections' observed pressures.
    b0 = h.rhs()
    rb0 = b0 - h.apply(x0)
    base_res = float(torch.linalg.norm(rb0) / torch.linalg.norm(b0))  # sign check of b - K x0
    u0 = x0.clone()
    u0[h.nf:] = 0
    y0 = h.apply(u0)
    nf = h.nf

    def correction(v, sigma):
        s = torch.expm1(-sigma * 1e-6 * v)
        m = 2.0 ** np.ceil(np.log2(2 * float(s.abs().max())))
        h.set_log_permeability(base - torch.log(s + m))
        ya = h.apply(u0)
        r = rb0.clone()
        r[:nf] -= ya[:nf] - m * y0[:nf]
        h.set_log_permeability(base + sigma * 1e-6 * v)
        e = h.zeros()
        try:
            h.solve(b=r, x=e, mode="fp64", tol=CORR_TOL)
        except vemgpu.VemGpuError:
            pass  # the FP64 floor was reached before CORR_TOL: e is the last iterate
        return obs.pressure(e)

    rng = np.random.default_rng(args.seed + 14)
    ad, fd, fdc = [], [], []
    t0 = time.time()
    base = torch.tensor(th, dtype=torch.float64, device="cuda")
    r0 = obs.pressure(x0) - obs.data
    for _ in range(args.fd_directions):
        v = torch.tensor(rng.standard_normal(h.nc), device="cuda")
        v = v / torch.linalg.norm(v)
        h.set_log_permeability(base + 1e-6 * v)
        jp = float(obs(solve_tight(x0)[0]))
        h.set_log_permeability(base - 1e-6 * v)
        jm = float(obs(solve_tight(x0)[0]))
        dp = correction(v, 1.0)
        dm = correction(v, -1.0)
        ad.append(float(grad @ v))
        fd.append((jp - jm) / 2e-6)
        fdc.append(float(((dp - dm) * (2 * r0 + dp + dm)).sum()) / 2e-6)
    h.set_log_permeability(base)
    ad, fd, fdc = np.array(ad), np.array(fd), np.array(fdc)
    # rounding floor of a central difference of J: one unit in the last place of J in each of the
    # two values, divided by 2 step; relative to the largest directional derivative
    ulp = float(np.spacing(abs(J)))
    floor = ulp / 2e-6 / np.abs(ad).max()
    err = float(np.abs(ad - fd).max() / np.abs(ad).max())
    out["fd_check"] = {"directions": len(ad), "step": 1e-6, "solve_tol": FD_TOL,
                       "max_abs_diff_over_max_abs_derivative": err,
                       "max_abs_diff_over_grad_norm": float(np.abs(ad - fd).max() / gn),
                       "rounding_floor_over_max_abs_derivative": floor, "error_in_floor_units": err / floor,
                       "max_abs_derivative": float(np.abs(ad).max()), "seconds": time.time() - t0,
                       "difference_form": {
                           "max_abs_diff_over_max_abs_derivative": float(np.abs(ad - fdc).max() / np.abs(ad).max()),
                           "correction_tol": CORR_TOL, "base_residual_b_minus_Kx0": base_res,
                           "how": "numerator J(+) - J(-) = sum_o (p+ - p-)(p+ + p- - 2 d_o) from the pressure "
                                  "corrections e = x(theta +- step v) - x0, each an FP64 solve of "
                                  "K(theta +- step v) e = b - K(theta) x0 - (K(theta +- step v) - K(theta)) x0, "
                                  "the last term formed from the per-cell scaling of the flux block"}}
    h.close()
    return out


def assembled_leg(g, z32, z64, stream_ms):
    """Comparator: the same operator assembled (vg_assemble_csr, the reference's assembled path) and
    multiplied by cuSPARSE (torch CSR SpMV), FP64 and FP32, timed like the matrix-free apply."""
    import torch
    t0 = time.time()
    C64 = g.assemble_csr(constrained=True)
    t_asm = time.time() - t0
    C32 = torch.sparse_csr_tensor(C64.crow_indices(), C64.col_indices(), C64.values().float(), size=C64.shape)
    nnz = int(C64.values().numel())
    spmv64 = stream_ms(lambda: torch.mv(C64, z64))
    spmv32 = stream_ms(lambda: torch.mv(C32, z32))
    out = {"nnz": nnz, "assemble_s": t_asm, "spmv_fp64_ms": spmv64, "spmv_fp32_ms": spmv32,
           "csr_bytes_fp64": nnz * 12 + 8 * (g.N + 1), "library": "cuSPARSE (torch CSR SpMV)"}
    del C64, C32
    torch.cuda.empty_cache()
    return out


def ms_leg(args):
    """Ternary Maxwell-Stefan on the 250k-cell disk: D12 = 1, D13 = 0.5, D23 = 0.2, seeded smooth
    initial fractions in [0.1, 0.8] summing to 1, backward Euler dt = 1e-3, 100 steps, each step
    fully implicit: Picard iterations on the friction matrix to relative change 1e-9 (the
    reference's default --picard-tol), every linear system to 1e-10; FP64 and FP32-refined runs,
    sum-to-one, bounds and species masses checked every step. One untimed step per precision
    first (the preconditioner build and graph capture of the first call, reported as
    first_call_step_s)."""
    import numpy as np
    import torch
    from vemgpu.maxwell_stefan import MaxwellStefan, initial_fractions
    mesh = disk_mesh(args.config1_cells, args.seed)
    ms = MaxwellStefan(mesh, D=(1.0, 0.5, 0.2), dt=1e-3, picard=50, picard_tol=1e-9)
    x1, x2, _ = initial_fractions(mesh, seed=args.seed + 31)
    s0 = ms.state(x1, x2)
    m0 = ms.masses(s0)
    out = {"cells": ms.nc, "unknowns": ms.N, "steps": args.ms_steps, "dt": 1e-3, "D": [1.0, 0.5, 0.2],
           "step": "backward Euler, fully implicit by Picard iterations on the friction matrix (tol 1e-9)"}
    finals = {}
    for mode in ("fp64", "mixed"):
        # untimed first step from the same state: the handle builds the species' multigrid from the
        # first stepped state (host aggregation) and captures this precision's Arnoldi graph on its
        # first call; the timed steps below start again from s0 with both in place
        _, winfo = ms.step(s0.clone(), mode=mode, tol=1e-10, inner_tol=1e-5)
        s = s0.clone()
        gs0 = ms.gram_schmidt_info()
        its, secs, pics, sum_err, mass_err, lo, hi = [], [], [], 0.0, 0.0, 1.0, 0.0
        for _ in range(args.ms_steps):
            s, info = ms.step(s, mode=mode, tol=1e-10, inner_tol=1e-5)
            its.append(info["iterations"])
            pics.append(info["picard"])
            secs.append(info["seconds"])
            f = ms.fractions(s)
            sum_err = max(sum_err, float(torch.abs(f[0] + f[1] + f[2] - 1).max()))
            lo = min(lo, min(float(x.min()) for x in f))
            hi = max(hi, max(float(x.max()) for x in f))
            mass_err = max(mass_err, max(abs(a - b) / abs(b) for a, b in zip(ms.masses(s), m0)))
        finals[mode] = torch.cat(ms.fractions(s)[:2])
        gs1 = ms.gram_schmidt_info()
        out[mode] = {"total_s": float(np.sum(secs)), "step_ms_mean": 1e3 * float(np.mean(secs)),
                     "iterations_mean": float(np.mean(its)), "iterations_max": int(np.max(its)),
                     "picard_mean": float(np.mean(pics)), "picard_max": int(np.max(pics)),
                     "max_sum_to_one_error": sum_err, "max_rel_mass_change": mass_err, "min_fraction": lo,
                     "max_fraction": hi, "first_call_step_s": winfo["seconds"],
                     "arnoldi_steps": gs1["arnoldi_steps"] - gs0["arnoldi_steps"],
                     "second_gram_schmidt_passes": gs1["reorthogonalizations"] - gs0["reorthogonalizations"]}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["total_s"] / out["mixed"]["total_s"]
    out["final_rel_diff_mixed_vs_fp64"] = float(torch.linalg.norm(finals["mixed"] - finals["fp64"]) /
                                                torch.linalg.norm(finals["fp64"]))
    ms.close()
    return out


def same_size_leg(args):
    """CPU reference algorithm and GPU solver on the same mesh: the --cpu-sample-cells annulus of
    the workload's family (same generator, seed and log-permeability field as the workload). CPU:
    assembly on one core and on all cores, GMRES(100)+ILU(0) to 1e-10 on one core, measured. GPU:
    handle set-up (mesh processing, device set-up kernels, multigrid) by wall clock, FP64 and mixed
    solves to 1e-10 by device time, and the end-to-end host-buffer solve."""
    import vemgpu
    mesh, _ = annulus_problem(args.cpu_sample_cells, args.seed)
    from vemgpu import fields
    theta = fields.gaussian_field(fields.cell_centroids(mesh), sigma=2.0, corr=0.1, seed=replica_seed(args.seed, 0))
    cells = len(mesh["cell_ptr"]) - 1
    out = {"cells": cells, "cpu": cpu_info()}
    for name, threads in (("cpu_1core", 1), ("cpu_allcore", os.cpu_count() or 1)):
        _, it, tm = cpu_solve(mesh, theta, threads)
        out[name] = {"assembly_s": tm["assembly_s"], "gmres_ilu_s": tm["solve_s"], "iterations": it,
                     "assembly_threads": threads}
    t0 = time.time()
    g = vemgpu.DarcyGpu(mesh, k=0, nq=9, ng=9, geometry="arcs", problem="annulus", bc="pressure", theta=theta)
    b = g.rhs()
    import torch
    torch.cuda.synchronize()
    out["gpu_setup_s"] = time.time() - t0
    for mode in ("fp64", "mixed"):
        g.solve(b, mode=mode, tol=1e-10, inner_tol=INNER_TOL)
        ts = [g.solve(b, mode=mode, tol=1e-10, inner_tol=INNER_TOL)[1]["seconds"] for _ in range(5)]
        out[f"gpu_{mode}_solve_s"] = sum(ts) / len(ts)
    bh = b.cpu().numpy()
    g.solve_host(bh, mode="mixed", tol=1e-10, inner_tol=INNER_TOL)
    t0 = time.perf_counter()
    for _ in range(5):
        g.solve_host(bh, mode="mixed", tol=1e-10, inner_tol=INNER_TOL)
    out["gpu_mixed_e2e_s"] = (time.perf_counter() - t0) / 5
    g.close()
    c1 = out["cpu_1core"]
    out["ratio_solve_vs_mixed"] = c1["gmres_ilu_s"] / out["gpu_mixed_solve_s"]
    out["ratio_solve_vs_fp64"] = c1["gmres_ilu_s"] / out["gpu_fp64_solve_s"]
    out["ratio_e2e"] = (c1["assembly_s"] + c1["gmres_ilu_s"]) / out["gpu_mixed_e2e_s"]
    out["ratio_setup_plus_solve"] = (out["cpu_allcore"]["assembly_s"] + out["cpu_allcore"]["gmres_ilu_s"]) / (
        out["gpu_setup_s"] + out["gpu_mixed_solve_s"])
    return out


def c1_leg(args):
    """Config C1: the 1,000-cell Voronoi disk, k = 0, K = I, p = sin(pi x) sin(pi y), Dirichlet
    pressure. CPU: the reference algorithm restated in the oracle (assembly + GMRES(100)+ILU(0),
    rtol 1e-10, one core), timed, with its flux and pressure L2 errors (the figures the reference
    prints per run, vem/CurvedVEM_Darcy/main/Darcy_curved_main.cpp:84-92) and the oracle's sparse-LU
    solution; GPU: FP64 and mixed solves to PARITY_TOL with the same figures and their relative
    distance to the LU solution."""
    import numpy as np
    import oracle as O
    import vemgpu
    mesh = disk_mesh(1000, args.seed)
    o = O.Oracle(mesh, k=0, nq=9, ng=9, geom=O.GEOM_ARCS, problem=O.PROB_SINSIN, bc=O.BC_PRESSURE)
    xo, _, _ = o.solve_direct()
    e_lu = o.errors(xo)
    xr, it, tm = cpu_solve(mesh, None, 1, problem=O.PROB_SINSIN)
    e_cpu = o.errors(xr)
    out = {"cells": o.nc, "dofs": o.N,
           "cpu_reference": {"seconds": tm["assembly_s"] + tm["solve_s"], "iterations": it, "residual": tm["rel"],
                             "l2_pressure": e_cpu["scalar_comp"], "l2_flux": e_cpu["flux_comp"],
                             "l2_pressure_phys": e_cpu["scalar_phys"], "l2_flux_phys": e_cpu["flux_phys"],
                             "rel_err_vs_lu": float(np.linalg.norm(xr - xo) / np.linalg.norm(xo))},
           "oracle_lu": {"l2_pressure": e_lu["scalar_comp"], "l2_flux": e_lu["flux_comp"]}}
    g = vemgpu.DarcyGpu(mesh, k=0, geometry="arcs", problem="sinsin", bc="pressure")
    for mode in ("fp64", "mixed"):
        g.solve(tol=PARITY_TOL, mode=mode, inner_tol=INNER_TOL)
        x, info = g.solve(tol=PARITY_TOL, mode=mode, inner_tol=INNER_TOL)
        e = g.errors(x)
        xg = x.cpu().numpy()
        out[mode] = {"solve_s": info["seconds"], "iterations": info["iterations"], "residual": info["residual"],
                     "rel_err_vs_lu": float(np.linalg.norm(xg - xo) / np.linalg.norm(xo)),
                     "l2_pressure": e["scalar_comp"], "l2_flux": e["flux_comp"]}
    g.close()
    return out


def c2_leg(args, job):
    """Config C2: the 250,000-cell disk of C1's problem, k = 0 and k = 1, FP64 and mixed solves to
    relative residual 1e-10 (device time) with the L2 errors against the manufactured solution,
    and the solves to PARITY_TOL compared with the oracle: for k = 0 the relative distance to the
    oracle's sparse-LU solution, for k = 1 the oracle's own residual ||b - K x|| / ||b|| of the GPU
    solution (the spawned check `job`, which ran beside the GPU legs)."""
    import numpy as np
    import vemgpu
    mesh = disk_mesh(args.config1_cells, args.seed)
    out = {"cells": len(mesh["cell_ptr"]) - 1}
    xo = None
    if job is not None:
        r = job.recv()
        xo = r["x"]
        out["oracle_lu_k0"] = {"seconds": r["seconds"], "l2_pressure": r["errors"]["scalar_comp"],
                               "l2_flux": r["errors"]["flux_comp"]}
    for k in (0, 1):
        g = vemgpu.DarcyGpu(mesh, k=k, geometry="arcs", problem="sinsin", bc="pressure")
        row = {"dofs": g.N}
        for mode in ("fp64", "mixed"):
            g.solve(tol=1e-10, mode=mode, inner_tol=INNER_TOL)
            x, info = g.solve(tol=1e-10, mode=mode, inner_tol=INNER_TOL)
            row[mode] = {"solve_s": info["seconds"], "iterations": info["iterations"], "residual": info["residual"]}
            xp, infop = g.solve(tol=PARITY_TOL, mode=mode, inner_tol=INNER_TOL)
            row[mode].update(parity_solve_s=infop["seconds"], parity_residual=infop["residual"])
            if k == 0 and xo is not None:
                xg = xp.cpu().numpy()
                row[mode]["rel_err_vs_oracle_lu"] = float(np.linalg.norm(xg - xo) / np.linalg.norm(xo))
                row[mode]["rel_err_vs_oracle_lu_at_1e-10"] = float(np.linalg.norm(x.cpu().numpy() - xo) /
                                                                   np.linalg.norm(xo))
        e = g.errors(x)
        row["l2_pressure"], row["l2_flux"] = e["scalar_phys"], e["flux_phys"]
        if k == 1 and job is not None:
            job.send(xp.cpu().numpy())
            r = job.recv()
            ep = g.errors(xp)
            row["oracle_residual_of_gpu_solution"] = r["residual"]
            row["oracle_vs_gpu_l2_pressure_rel"] = abs(r["errors"]["scalar_phys"] / ep["scalar_phys"] - 1)
        out[f"k{k}"] = row
        g.close()
    if job is not None:
        job.close()
    return out


def max_over_ranks(value, dist):
    """The largest value over all ranks (every rank calls this at the same point); the tensor lives
    on the GPU for NCCL and on the host for gloo."""
    if not dist:
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(seed, rank):
    """Seed of the permeability field of one replica: replicas solve different fields of the same
    workload (same mesh, no data exchanged between ranks)."""
    return seed + 1 + rank


def ours(args, rank, world, dist):
    import numpy as np
    import torch
    import vemgpu

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # rank 0 builds the mesh cache; replicas differ by their permeability seed
    if rank == 0:
        annulus_problem(args.cells, args.seed)
    if dist:
        dist.barrier()
    mesh, _ = annulus_problem(args.cells, args.seed)
    from vemgpu import fields
    theta = fields.gaussian_field(fields.cell_centroids(mesh), sigma=2.0, corr=0.1, seed=replica_seed(args.seed, rank))
    # the oracle's CPU checks of configs C2 and C4 (sparse LU of 1M-unknown systems, minutes of one
    # core each) run in spawned processes beside the GPU legs; rank 0 of a single-GPU run only
    jobs = {}
    if rank == 0 and world == 1 and not args.profile and not args.no_oracle_checks:
        if not args.no_config1:
            disk_mesh(args.config1_cells, args.seed)
            jobs["c2"] = OracleJob("c2", os.path.join(CACHE, f"disk_{args.config1_cells}_s{args.seed}.npz"))
        if not args.no_adjoint:
            amesh, _ = annulus_problem(args.adjoint_cells, args.seed)
            ath = fields.gaussian_field(fields.cell_centroids(amesh), sigma=2.0, corr=0.1, seed=args.seed + 11)
            jobs["c4"] = OracleJob("c4", os.path.join(CACHE, f"annulus_{args.adjoint_cells}_s{args.seed}.npz"), ath)
    t0 = time.time()
    g = vemgpu.DarcyGpu(mesh, k=0, nq=9, ng=9, geometry="arcs", problem="annulus", bc="pressure", theta=theta)
    setup_s = time.time() - t0
    b = g.rhs()
    x = g.zeros()
    if args.profile:
        # fixed sequence for profilers: 5 FP32 applies, 5 FP64 applies, one FP64 and one mixed solve
        z = torch.randn(g.N, dtype=torch.float32, device="cuda")
        y = torch.empty_like(z)
        for _ in range(5):
            g.apply(z, out=y)
        z64, y64 = z.double(), y.double()
        for _ in range(5):
            g.apply(z64, out=y64)
        ce = 16 if args.eager else 0
        g.solve(b, x, mode="fp64", tol=1e-10, check_every=ce)
        g.solve(b, x, mode="mixed", tol=1e-10, inner_tol=INNER_TOL, check_every=ce)
        torch.cuda.synchronize()
        if args.profile_ms:
            # Maxwell-Stefan kernels: 3 FP64 and 3 FP32 applies, one FP64 and one mixed step, on a
            # disk of the same cell count
            from vemgpu.maxwell_stefan import MaxwellStefan, initial_fractions
            dm = disk_mesh(args.cells, args.seed)
            ms = MaxwellStefan(dm, D=(1.0, 0.5, 0.2), dt=1e-3)
            x1, x2, _ = initial_fractions(dm, seed=args.seed + 31)
            st = ms.state(x1, x2)
            zz = torch.randn(ms.N, dtype=torch.float64, device="cuda")
            for _ in range(3):
                ms.apply(st, zz)
                ms.apply(st, zz.float())
            for mode in ("fp64", "mixed"):
                ms.step(st, mode=mode, tol=1e-10, inner_tol=1e-5)
            torch.cuda.synchronize()
            ms.close()
        print(json.dumps({"profile": "done", "cells": g.nc, "dofs": g.N}), flush=True)
        return

    def solve(mode):
        return g.solve(b, x, mode=mode, tol=1e-10, inner_tol=INNER_TOL)[1]

    def timed(mode, steps, warmup):
        for _ in range(warmup):
            solve(mode)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        infos = []
        l0 = g.stats()["launches"]
        e0.record()
        for _ in range(steps):
            infos.append(solve(mode))
        e1.record()
        torch.cuda.synchronize()
        launches = g.stats()["launches"] - l0
        if dist:
            dist.barrier()
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms, dist), infos, launches

    clk = ClockSampler(os.path.join(tempfile.gettempdir(), f"vg_clocks_{os.getpid()}.csv"))
    with clk:
        ms_mixed, info_mixed, launches = timed("mixed", args.steps, args.warmup)
    clocks = clk.summary(local)
    x_mixed = x.clone()
    res = {}
    if not args.no_fp64 and not args.profile:
        ms64, info64, _ = timed("fp64", max(1, args.steps // 2), 1)
        res["fp64"] = dict(solve_s=ms64 * 1e-3, iterations=info64[0]["iterations"], residual=info64[0]["residual"],
                           speedup_mixed_vs_fp64=ms64 / ms_mixed)
        x64 = x.clone()
        res["fp64"]["rel_diff_mixed_vs_fp64"] = float(torch.linalg.norm(x_mixed - x64) / torch.linalg.norm(x64))
        # FP64 reference of the 1M-cell workload (the oracle's sparse LU does not reach this size):
        # the FP64 solve driven to the FP64 floor, true residual 1e-14
        xr = g.zeros()
        try:
            _, ir = g.solve(b, xr, mode="fp64", tol=1e-14)
            ref_res = ir["residual"]
        except vemgpu.VemGpuError:
            ref_res = float("nan")
        nr = torch.linalg.norm(xr)
        res["accuracy"] = {"reference": "FP64 GPU solve to true relative residual 1e-14",
                           "reference_residual": ref_res,
                           "mixed_rel_err": float(torch.linalg.norm(x_mixed - xr) / nr),
                           "fp64_rel_err": float(torch.linalg.norm(x64 - xr) / nr), "target": 1e-10}
        del xr
    # per-kernel device times on the same buffers (FP32 apply, FP64 apply) with L2 flushed in between
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    z32 = torch.randn(g.N, dtype=torch.float32, device="cuda")
    z64 = z32.double()

    def kernel_ms(fn, reps=20):
        tot = 0.0
        for _ in range(3):
            fn()
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    y32, y64 = torch.empty_like(z32), torch.empty_like(z64)

    def stream_ms(fn, reps=40):
        # back-to-back launches: the operator stream (> 126 MB) does not fit L2 between launches
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # the kernel as the solver runs it: vectors in the solver's internal order (vg_apply with
    # VG_ORDER_INTERNAL, no permutation); vg_apply zeroes y before the kernel (the solver's loop
    # zeroes it inside the update kernel), so the kernel's own time is the back-to-back apply time
    # less the back-to-back memset time
    zi32, zi64 = g.permute(z32), g.permute(z64)
    apply32_ms = (stream_ms(lambda: g.apply(zi32, out=y32, internal_order=True)) -
                  stream_ms(lambda: y32.zero_()))
    apply64_ms = (stream_ms(lambda: g.apply(zi64, out=y64, internal_order=True)) -
                  stream_ms(lambda: y64.zero_()))
    apply32_public_ms = stream_ms(lambda: g.apply(z32, out=y32))
    apply64_public_ms = stream_ms(lambda: g.apply(z64, out=y64))
    assembled = None if args.no_assembled else assembled_leg(g, z32, z64, stream_ms)
    apply32_flushed_ms = kernel_ms(lambda: g.apply(zi32, out=y32, internal_order=True))
    apply64_flushed_ms = kernel_ms(lambda: g.apply(zi64, out=y64, internal_order=True))
    b32, b64 = apply_bytes(g, mesh, 32), apply_bytes(g, mesh, 64)
    peak, peak_kind = peaks()
    ach32 = b32 / (apply32_ms * 1e-3) / 1e9
    ach64 = b64 / (apply64_ms * 1e-3) / 1e9
    # end to end through the host-buffer C ABI call (H2D of b and D2H of x inside)
    bh_t = torch.empty(g.N, dtype=torch.float64, pin_memory=True)
    bh_t.copy_(b)
    xh_t = torch.empty(g.N, dtype=torch.float64, pin_memory=True)
    bh, xh = bh_t.numpy(), xh_t.numpy()
    e2e = []
    for i in range(1 + args.steps):
        t = time.perf_counter()
        _, info_h = g.solve_host(bh, out=xh, mode="mixed", tol=1e-10, inner_tol=INNER_TOL)
        if i:
            e2e.append(time.perf_counter() - t)
    e2e_s = max_over_ranks(sum(e2e) / len(e2e), dist)
    adjoint = None if args.no_adjoint else adjoint_leg(args, rank, jobs.get("c4"))
    config1 = None if args.no_config1 else c2_leg(args, jobs.get("c2"))
    c1 = None if args.no_config1 else c1_leg(args)
    ms = None if args.no_ms else ms_leg(args)
    cpu = same = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile:
        same = same_size_leg(args)
        one = same["cpu_1core"]
        cpu = {"value": one["assembly_s"] + one["gmres_ilu_s"], "unit": "s", "cores": 1, "kind": "port",
               "cells": same["cells"],
               "sample": f"reference algorithm restated (oracle): element matrices, CSR assembly, GMRES(100)+ILU(0) "
                         f"rtol 1e-10 on one core, measured per solve on a {same['cells']}-cell annulus of the "
                         f"workload's family (not scaled; the same mesh solved on the GPU in same_size: "
                         f"{same['ratio_solve_vs_mixed']:.0f}x); CPU {same['cpu']['model']}"}
    if rank != 0:
        return
    contrast = float(np.exp(theta.max() - theta.min()))
    line = {
        "metric": METRIC, "value": ms_mixed * 1e-3, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"annulus 0.3<r<1, {g.nc} Voronoi+Lloyd cells (exact arcs), k=0, lognormal K "
                               f"(sigma 2, corr 0.1, K max/min {contrast:.2e}), p=1 inner / 0 outer, FP32 inner "
                               f"MINRES + FP64 refinement to ||b-Ax||/||b|| <= 1e-10",
                   "cells": g.nc, "edges": g.ne, "dofs": g.N, "k": 0, "nq": 9, "ng": 9,
                   "l2": "inputs larger than L2: every MINRES iteration streams the operator (144 MB FP32, "
                         "261 MB FP64) and the multigrid hierarchy; apply timings back to back (operator > L2) "
                         "and with L2 flushed", "parallelism": f"replicas x{world}"},
        "throughput": {"solves_per_s": world / (ms_mixed * 1e-3), "replicas": world},
        "iterations": info_mixed[0]["iterations"], "outer": info_mixed[0]["outer"],
        "residual": info_mixed[0]["residual"], "setup_s": setup_s, "fp64": res.get("fp64"),
        "accuracy": res.get("accuracy"),
        "kernels": {"apply_fp32_ms": apply32_ms, "apply_fp64_ms": apply64_ms, "apply_fp32_bytes": b32,
                    "apply_fp64_bytes": b64, "apply_fp32_flushed_ms": apply32_flushed_ms,
                    "apply_fp64_flushed_ms": apply64_flushed_ms,
                    "vg_apply_reference_order_fp32_ms": apply32_public_ms,
                    "vg_apply_reference_order_fp64_ms": apply64_public_ms},
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
                     "traffic": traffic_bytes("apply_bulk_kernel<float, 0>", g.nc),
                     "kernel": "apply_bulk_kernel<float, 0> (FP32 matrix-free apply, bulk-copied piece records)",
                     "peak_kind": peak_kind, "fp64_apply_frac": ach64 / peak,
                     "fp64_traffic": traffic_bytes("apply_bulk_kernel<double, 0>", g.nc)},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * g.N, "d2h_bytes_per_step": 8 * g.N},
        "assembled_comparator": assembled,
        "adjoint": adjoint,
        "disk_250k": config1,
        "disk_1k": c1,
        "maxwell_stefan": ms,
        "same_size": same,
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    line["summary"] = summary(line)  # last: the figures a reader of the line's end needs
    print(json.dumps(line), flush=True)


def summary(line):
    """The headline figures of every leg in a few keys (the end of the JSON line)."""
    def get(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or d.get(k) is None:
                return None
            d = d[k]
        return d

    def r(v, n=3):
        return None if v is None else float(f"{v:.{n}g}")
    f = line.get("fp64") or {}
    out = {"mixed_s": r(line["value"]), "fp64_s": r(f.get("solve_s")),
           "mixed_over_fp64": r(f.get("speedup_mixed_vs_fp64")),
           "mixed_err_vs_fp64_ref": r(get(line, "accuracy", "mixed_rel_err")),
           "apply_fp32_frac": r(line["roofline"]["frac"]), "apply_fp64_frac": r(line["roofline"]["fp64_apply_frac"]),
           "e2e_s": r(line["e2e"]["value"])}
    a = line.get("adjoint")
    if a:
        out.update(grad_over_solve=r(get(a, "mixed", "grad_over_solve")),
                   grad_vs_cpu=r(get(a, "cpu_gradient", "max_abs_diff_over_max_abs")),
                   fd_vs_max_derivative=r(get(a, "fd_check", "max_abs_diff_over_max_abs_derivative")),
                   fd_difference_form=r(get(a, "fd_check", "difference_form", "max_abs_diff_over_max_abs_derivative")),
                   fd_floor=r(get(a, "fd_check", "rounding_floor_over_max_abs_derivative")))
    c2 = line.get("disk_250k")
    if c2:
        out.update(c2_k0_err_vs_lu=r(get(c2, "k0", "mixed", "rel_err_vs_oracle_lu_at_1e-10")),
                   c2_k1_oracle_residual=r(get(c2, "k1", "oracle_residual_of_gpu_solution")))
    c1 = line.get("disk_1k")
    if c1:
        out.update(c1_err_vs_lu=r(get(c1, "mixed", "rel_err_vs_lu")), c1_cpu_s=r(get(c1, "cpu_reference", "seconds")),
                   c1_l2_p=r(get(c1, "cpu_reference", "l2_pressure")), c1_l2_u=r(get(c1, "cpu_reference", "l2_flux")))
    ss = line.get("same_size")
    if ss:
        out.update(same_size_cells=ss["cells"], same_size_cpu_over_gpu_solve=r(ss["ratio_solve_vs_mixed"]),
                   same_size_cpu_over_gpu_e2e=r(ss["ratio_e2e"]))
    ms = line.get("maxwell_stefan")
    if ms:
        out.update(ms_mixed_s=r(get(ms, "mixed", "total_s")), ms_fp64_s=r(get(ms, "fp64", "total_s")))
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        ours(args, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
