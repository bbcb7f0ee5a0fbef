"""Benchmark: icosphere-L8 Helmholtz solves per second to 1e-8 relative residual on B200.

Workload (one "step"): a batch of 32 Helmholtz solves (L + I) u = b on the icosphere L8
(655,362 vertices, 1,310,720 triangles; unit icosahedron binary-subdivided 8 times with the new
vertices projected to the unit sphere, circumcentric duals), b_j uniform[-1, 1] (seeds 2..33),
each solved to ‖b - A u‖ / ‖b‖ ≤ 1e-8 by FP32 V-cycles inside FP64 iterative refinement
(Chebyshev-Jacobi smoother, dense FP64 coarsest solve).  `value` times the solve with b
resident in HBM (168 MB of FP64 right-hand sides per step, more than the 126 MB L2); `e2e`
times the same solve through the C ABI with host buffers, the copies inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun, one process per GPU): every rank solves its own batch (seeds offset by rank);
there is no data-path collective ("scaling": "weak"); rank 0 prints the max-over-ranks time.
`--impl reference` times the reference algorithm (Multigrid.jl V-cycles with the Krylov CG
smoother, FP64) on the host cores through the CPU oracle, on rank 0 only.
"""
import argparse
import importlib.util
import json
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
LEVEL = 8
NRHS = 32
RTOL = 1e-8
SHIFT = 1.0


def load_package():
    if "dec_b200" in sys.modules:
        return sys.modules["dec_b200"]
    pkg = ROOT / "combinatorialspaces.jl_b200"
    spec = importlib.util.spec_from_file_location("dec_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dec_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        v = d.get(kernel)
        if isinstance(v, dict):
            return v.get("bytes_per_launch")
        return v
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.lines = []
        self.device = device_index

    def start(self):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            ident = ["-i", uuid if uuid.startswith("GPU-") else "GPU-" + uuid]
        except Exception:
            ident = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", *ident, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_operator_baseline(reps=100):
    """The plain-operator workload on the host cores: the oracle's statement of the reference's CPU
    kernels (FastDEC's wedge kernels, SparseArrays' products) on the 128 x 128 grid, µs per operation,
    on one thread and on every host thread (a thread per slice of rows, started per call)."""
    sys.path.insert(0, str(ROOT))
    import oracle
    O = oracle.load()
    m = O.triangulated_grid(127, 127, 1.0, 1.0, compress=False)
    d = O.dualize(m, O.BARYCENTER)
    dec = load_package()
    f, a, b = dec.meshes.uniform(0, d.nv), dec.meshes.uniform(1, d.ne), dec.meshes.uniform(2, d.ne)
    out = {}
    for threads in sorted({1, os.cpu_count() or 1}):
        O.set_num_threads(threads)
        t = O.time_operators(d, f, a, b, reps)
        out[f"{threads}_threads"] = {"wedge01(f,alpha)": round(t["wedge01"] * 1e6, 2),
                                     "wedge11(alpha,beta)": round(t["wedge11"] * 1e6, 2),
                                     "wedge02(f,d1 alpha)": round(t["wedge02_d1"] * 1e6, 2),
                                     "laplacian f": round(t["laplacian"] * 1e6, 2)}
    O.set_num_threads(1)
    out["kind"] = "port (the oracle's C++ statement, -O2; µs per operation, mean of 100 after one warm-up)"
    return out


def measure_operators(dec, peak, cpu=True):
    """HBM roofline of the DEC operator kernels: each kernel timed alone with CUDA events, L2
    flushed before every launch by reading a 256 MB buffer (a read leaves L2 holding clean lines,
    so the timed kernel pays no write-back of the flush), on icosphere L9 (circumcentric duals) and a
    2049x2049 grid (barycentric duals, a 9x9 triangulated grid binary-refined 8 times), FP64 and
    FP32.  Algorithmic bytes: every streamed array once, each gathered form once (int32 indices)."""
    import torch

    flush = torch.ones(64 * 2 ** 20, dtype=torch.float32, device="cuda")
    sink = torch.empty((), dtype=torch.float32, device="cuda")

    def time_op(fn, reps=10):
        fn()
        tot = 0.0
        for _ in range(reps):
            torch.sum(flush, dim=0, out=sink)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    big_grid = dec.meshes.triangulated_grid(8, 8, 1.0, 1.0, False)
    for _ in range(8):
        big_grid = dec.meshes.refine_binary(big_grid)
    cases = [("icosphere_L9", dec.meshes.icosphere(9), "circumcenter"), ("grid_2049x2049", big_grid, "barycenter")]
    out = {}
    for name, m, center in cases:
        g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                     center=center)
        nv, ne, nt = g.nv, g.ne, g.nt
        width = int(np.bincount(np.concatenate([m.ev0, m.ev1]), minlength=nv).max()) + 1
        res = {"nv": nv, "ne": ne, "nt": nt}
        for dt, tdt, sz in (("float64", torch.float64, 8), ("float32", torch.float32, 4)):
            f = torch.rand(nv, dtype=tdt, device="cuda")
            a = torch.rand(ne, dtype=tdt, device="cuda")
            b = torch.rand(ne, dtype=tdt, device="cuda")
            tt = torch.rand(nt, dtype=tdt, device="cuda")
            oe = torch.empty(ne, dtype=tdt, device="cuda")
            ot = torch.empty(nt, dtype=tdt, device="cuda")
            ov = torch.empty(nv, dtype=tdt, device="cuda")
            w01 = dec.dec_wedge_product(0, 1, g, dt)
            w11 = dec.dec_wedge_product(1, 1, g, dt)
            w02 = dec.dec_wedge_product(0, 2, g, dt)
            d0 = dec.dec_differential(0, g, dt)
            d1 = dec.dec_differential(1, g, dt)
            L = dec.laplace_beltrami(g, dt)
            ell_rows = L.autotune(reps=10)   # rows per thread of the ELL apply, recorded in the tuning table
            s1 = dec.hodge_operator(1, g, dtype=dt)
            ops = {
                "wedge01": (lambda: w01(f, a, oe), ne * (8 + 2 * sz) + nv * sz),
                "wedge11": (lambda: w11(a, b, ot), nt * (12 + 4 * sz) + 2 * ne * sz),
                "wedge02": (lambda: w02(f, tt, ot), nt * (12 + 5 * sz) + nv * sz),
                "d0": (lambda: d0.apply(f, oe), ne * (9 + sz) + nv * sz),
                "d1": (lambda: d1.apply(a, ot), nt * (13 + sz) + ne * sz),
                "laplacian": (lambda: L.apply(f, ov), nv * width * (4 + sz) + 2 * nv * sz),
                "star1": (lambda: s1.apply(a, oe), 3 * ne * sz),
            }
            for op, (fn, by) in ops.items():
                ms = time_op(fn)
                gbs = by / (ms * 1e-3) / 1e9
                res[f"{op}_{dt}"] = {"us": round(ms * 1e3, 2), "GB/s": round(gbs, 1), "frac": round(gbs / peak, 3)}
                if op == "laplacian":
                    res[f"{op}_{dt}"]["rows_per_thread"] = ell_rows
        out[name] = res
        del g
        torch.cuda.empty_cache()

    # The plain-operator workload: the 128 x 128 grid, barycentric duals, FP64, 100 repetitions of
    # each operation (L2-resident: µs per operation, not an HBM figure).
    m = dec.meshes.triangulated_grid(127, 127, 1.0, 1.0, False)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                 center="barycenter")
    f = torch.tensor(dec.meshes.uniform(0, g.nv), device="cuda")
    al = torch.tensor(dec.meshes.uniform(1, g.ne), device="cuda")
    be = torch.tensor(dec.meshes.uniform(2, g.ne), device="cuda")
    w01, w11, w02 = (dec.dec_wedge_product(0, 1, g), dec.dec_wedge_product(1, 1, g),
                     dec.dec_wedge_product(0, 2, g))
    d1, L = dec.dec_differential(1, g), dec.laplace_beltrami(g)
    d1a = torch.empty(g.nt, dtype=torch.float64, device="cuda")
    o01 = torch.empty(g.ne, dtype=torch.float64, device="cuda")
    o11 = torch.empty(g.nt, dtype=torch.float64, device="cuda")
    o02 = torch.empty(g.nt, dtype=torch.float64, device="cuda")
    oL = torch.empty(g.nv, dtype=torch.float64, device="cuda")
    grid_ops, grid_graph = {}, {}
    for name, fn in (("wedge01(f,alpha)", lambda: w01(f, al, o01)), ("wedge11(alpha,beta)", lambda: w11(al, be, o11)),
                     ("wedge02(f,d1 alpha)", lambda: w02(f, d1.apply(al, d1a), o02)),
                     ("laplacian f", lambda: L.apply(f, oL))):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(100):
            fn()
        e1.record()
        torch.cuda.synchronize()
        grid_ops[name] = round(e0.elapsed_time(e1) * 10, 2)  # µs per op (ms / 100 * 1000)
        # the same 100 repetitions captured in one CUDA graph: the device time per operation
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr):
            for _ in range(100):
                fn()
        gr.replay()
        torch.cuda.synchronize()
        e0.record()
        gr.replay()
        e1.record()
        torch.cuda.synchronize()
        grid_graph[name] = round(e0.elapsed_time(e1) * 10, 2)
        del gr
    out["grid_128x128_us_per_op"] = grid_ops
    out["grid_128x128_us_per_op_graph"] = grid_graph
    if cpu:
        out["grid_128x128_cpu_us_per_op"] = cpu_operator_baseline()
    return out


def training_tensor_flop(steps, batch=65536, levels=(5, 6, 7), block=10):
    """Tensor-core FLOP of `steps` training steps of learned.train_smoother's schedule: per step the
    forward over every sample of its fields (2·(16·64 + 64·64) = 10,240 per sample), and per batch
    sample the recomputed forward (10,240), dh1 = W2ᵀ dz2 with dz2 as two BF16 parts (2·2·64·64 =
    16,384) and the weight gradients with dz as two parts (dW2 16,384, dW1 4,096)."""
    n = {lv: 10 * 4 ** lv + 2 for lv in levels}
    per_step = {5: 6, 6: 2, 7: 1}
    total, t = 0.0, 0
    while t < steps:
        for lv in levels:
            if t >= steps:
                break
            nb = min(block, steps - t)
            N = n[lv] * per_step.get(lv, 1)
            total += nb * (N * 10240.0 + min(batch, N) * (10240.0 + 16384.0 + 16384.0 + 4096.0))
            t += nb
    return total


def run_train(args):
    """The learned smoother's training alone (the entry point for the training launch list)."""
    import torch
    dec = load_package()
    from dec_b200 import learned
    t0 = time.perf_counter()
    mlp, losses = learned.train_smoother(steps=args.train_steps, lr=1e-3, batch=65536, seed=4, shift=SHIFT)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    print(json.dumps({"train_steps": args.train_steps, "seconds": t, "final_loss": losses[-1][2],
                      "tensor_TFLOP": training_tensor_flop(args.train_steps) / 1e12}), flush=True)


def measure_learned(dec, args, B, U64, common, timed):
    """The learned smoother: trained on the GPU (Adam, lr 1e-3, batch 65,536 vertex samples, seed
    4) on V-cycle (residual, error) pairs of icospheres L5-L7, then used as the smoother at every
    level of FP32 V-cycles in FP64 refinement: on the L8 workload (against the FP64 solution
    U64) and on icosphere L9 (2,621,442 vertices) against the plain Chebyshev smoother, with
    the plain smoother as fallback."""
    import torch
    from dec_b200 import learned
    t0 = time.perf_counter()
    mlp, losses = learned.train_smoother(steps=args.train_steps, lr=1e-3, batch=65536, seed=4, shift=SHIFT)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    ico = dec.meshes.icosahedron()
    flop = training_tensor_flop(args.train_steps)
    out = {"train": {"steps": args.train_steps, "seconds": train_s, "final_losses": [round(l, 4) for _, _, l in losses[-3:]],
                     "tensor_TFLOP": flop / 1e12, "tensor_TFLOP/s_incl_setup": flop / train_s / 1e12,
                     "engine": "mma.sync m16n8k16 (forward, backward, weight gradients)"}}

    def run(level, smoother, sweeps, Bm, Uref=None, engine="tcgen05"):
        # the learned V(1,1) solve is fastest with 2 cycles per refinement step (measured 1, 2, 3)
        opts = dict(common, smoother=smoother, pre=sweeps, post=sweeps)
        if smoother == 3:
            opts["inner_cycles"] = 2
        mg = dec.MultigridData(ico, level, precision=1, **opts)
        if smoother == 3:
            mlp.set_engine(engine)
            mg.set_smoother_mlp(mlp)
        U = torch.zeros_like(Bm)

        def solve():
            return mg.solve(U, Bm, rtol=RTOL, max_iters=100, use_initial_guess=False)[1]

        t, reps = timed(solve, max(1, args.steps), 1)
        rep = reps[-1]
        res = {"solves_per_s": Bm.shape[0] * max(1, args.steps) / t, "refinement_steps": int(rep.iterations),
               "v_cycles_per_solve": int(rep.iterations) * opts.get("inner_cycles", common["inner_cycles"]),
               "converged": bool(rep.converged), "fallback_iteration": int(rep.fallback_iteration),
               "sweeps": sweeps}
        if smoother == 3:
            res["mlp_engine"] = engine
        if Uref is not None:
            res["max_rel_error_vs_fp64_solve"] = float(((U - Uref).norm(dim=1) / Uref.norm(dim=1)).max())
        if smoother == 3:
            ms, _ = mg.time_kernel(4, 0, Bm.shape[0], reps=5)
            nv = mg.level_info(0)[0]
            res["mlp_kernel_ms"] = ms
            res["mlp_tensor_tflops"] = 10240.0 * nv * Bm.shape[0] / (ms * 1e-3) / 1e12
        del mg
        torch.cuda.empty_cache()
        return res

    out["L8_learned_fp32"] = {f"V({k},{k})": run(LEVEL, 3, k, B, U64) for k in (1, 2)}
    out["L8_learned_fp32_mma_sync"] = {"V(1,1)": run(LEVEL, 3, 1, B, U64, engine="mma")}
    n9 = 10 * 4 ** 9 + 2
    B9 = torch.tensor(np.stack([dec.meshes.uniform(200 + j, n9) for j in range(NRHS)]), device="cuda")
    out["L9_learned_fp32"] = {f"V({k},{k})": run(9, 3, k, B9) for k in (1, 2)}
    out["L9_learned_fp32_mma_sync"] = {"V(1,1)": run(9, 3, 1, B9, engine="mma")}
    out["L9_plain_fp32"] = {f"V({k},{k})": run(9, 1, k, B9) for k in (2, 3)}
    del B9
    torch.cuda.empty_cache()
    return out


def measure_batched(dec, args):
    """The batched uneven workload: 512 Helmholtz solves (L + c I) u = b, c log-uniform in [0.1, 10]
    and the mesh drawn uniformly from 8 types (icospheres L4-L7; planar grids 65^2, 129^2, 257^2,
    513^2 = a 9x9 triangulated grid refined 3-6 times), seed 3; FP32 Chebyshev cycles (the headline's
    --pre / --post / --cheb-ratio / --inner-cycles) in
    FP64 refinement to 1e-8, every refinement step of all 8 groups one CUDA graph, panel widths
    per group from the autotuner.  Then 1,024 wedge products ∧(1,1) of FP32 uniform[-1,1] 1-form
    pairs on icosphere L7 in one batched launch."""
    import torch
    rng = np.random.default_rng(3)
    ico = dec.meshes.icosahedron()
    grid9 = dec.meshes.triangulated_grid(8, 8, 1.0, 1.0, False)
    types = [("icosphere_L4", ico, 4, 1.0), ("icosphere_L5", ico, 5, 1.0), ("icosphere_L6", ico, 6, 1.0),
             ("icosphere_L7", ico, 7, 1.0), ("grid_65x65", grid9, 3, 0.0), ("grid_129x129", grid9, 4, 0.0),
             ("grid_257x257", grid9, 5, 0.0), ("grid_513x513", grid9, 6, 0.0)]
    draw = rng.integers(0, len(types), 512)
    cs = np.exp(rng.uniform(np.log(0.1), np.log(10.0), 512))
    t0 = time.perf_counter()
    mgs, nrhs, shifts, Bs = [], [], [], []
    for t, (name, coarse, levels, radius) in enumerate(types):
        mg = dec.MultigridData(coarse, levels, shift=0.0, center="circumcenter", project_radius=radius,
                               smoother=1, pre=args.pre, post=args.post, cheb_ratio=args.cheb_ratio, precision=1,
                               coarse_solver=2, coarse_max=170, inner_cycles=args.inner_cycles)
        idx = np.nonzero(draw == t)[0]
        mgs.append(mg)
        nrhs.append(len(idx))
        shifts.append(cs[idx])
        Bs.append(torch.tensor(np.stack([dec.meshes.uniform(1000 + int(i), mg.n) for i in idx]), device="cuda"))
    batch = dec.Batch(mgs)
    batch.autotune(nrhs, reps=3)
    setup_s = time.perf_counter() - t0
    Us = [torch.zeros_like(B) for B in Bs]

    def solve():
        for U in Us:
            U.zero_()
        return batch.solve(Us, Bs, shifts=shifts, rtol=RTOL, max_iters=60)

    for _ in range(max(1, args.warmup)):
        solve()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = max(1, args.steps)
    e0.record()
    outs = [solve() for _ in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    reps, tot = outs[-1]
    groups = {}
    for (name, _, _, _), mg, r, k in zip(types, mgs, reps, nrhs):
        groups[name] = {"vertices": mg.n, "solves": k, "refinement_steps": int(r.iterations),
                        "converged": bool(r.converged), "panel_width": int(r.rhs_block)}
    peak, peak_kind = measured_peaks()
    by_batch = batch.traffic(int(tot.iterations))
    res = {"solves": 512, "solves_per_s": 512 * steps / t, "ms_per_batch": 1e3 * t / steps,
           "bytes_per_batch": by_batch, "GB/s": by_batch / (t / steps) / 1e9,
           "frac": by_batch / (t / steps) / 1e9 / peak, "peak": peak_kind,
           "refinement_steps": int(tot.iterations), "converged": bool(tot.converged),
           "max_rel_residual": tot.max_rel_residual, "kernels_per_batch": int(tot.launches),
           "setup_seconds": setup_s, "groups": groups}
    del Us, Bs, batch, mgs
    torch.cuda.empty_cache()

    # 1,024 wedge products on icosphere L7 (FP32), one batched launch
    m7 = dec.meshes.icosphere(7)
    g7 = dec.Mesh(m7.points, m7.ev0, m7.ev1, m7.te0, m7.te1, m7.te2, m7.edge_orientation, m7.tri_orientation,
                  center="circumcenter")
    ne, nt = g7.ne, g7.nt
    w11 = dec.dec_wedge_product(1, 1, g7, "float32")
    count = 1024
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    a = torch.rand((count, ne), dtype=torch.float32, device="cuda", generator=gen) * 2 - 1
    b = torch.rand((count, ne), dtype=torch.float32, device="cuda", generator=gen) * 2 - 1
    out = torch.empty((count, nt), dtype=torch.float32, device="cuda")
    pairs = w11.autotune(count, reps=3)  # form pairs per thread, from the project autotuner
    w11.batched(a, b, out)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        w11.batched(a, b, out)
    e1.record()
    torch.cuda.synchronize()
    tw = e0.elapsed_time(e1) / 1e3 / steps
    by = count * (2.0 * ne * 4 + nt * 4) + nt * (12 + 3 * 4)
    res["wedge11_L7_fp32_x1024"] = {"ms": 1e3 * tw, "wedges_per_s": count / tw, "GB/s": by / tw / 1e9,
                                    "bytes": by, "frac": by / tw / 1e9 / peak, "peak": peak_kind,
                                    "pairs_per_thread": pairs}
    del a, b, out
    torch.cuda.empty_cache()
    return res


def oracle_hierarchy(level, threads):
    """The oracle's icosphere hierarchy of `level` binary subdivisions (checker only: the errors the
    GPU results are stated against)."""
    sys.path.insert(0, str(ROOT))
    import oracle
    O = oracle.load()
    O.set_num_threads(threads)
    return oracle, O, O.build_mg(O.icosahedron(), level, O.CIRCUMCENTER, SHIFT, 1.0, 3)


def measure_config2(dec, args):
    """Plain FP64 multigrid on icosphere L6 (40,962 vertices): (L + I) u = b, b uniform[-1,1] with
    seed 1, V(3,3) Chebyshev-Jacobi cycles with a dense direct solve on L0 (12 vertices), to 1e-10
    relative residual.  GPU: the device refinement loop (FP64 V-cycles), one right-hand side and the
    32-RHS batch; the error is against the oracle's FP64 solve to 1e-13; the CPU figure is the same
    V-cycle in the oracle on all host threads."""
    import torch
    ico = dec.meshes.icosahedron()
    mg = dec.MultigridData(ico, 6, shift=SHIFT, center="circumcenter", project_radius=1.0, precision=0,
                           smoother=1, pre=3, post=3, cheb_ratio=4.0, coarse_solver=0, coarse_max=0)
    n = mg.n
    b = torch.tensor(dec.meshes.uniform(1, n), device="cuda")
    U = torch.zeros_like(b)
    steps = max(3, args.steps)

    def rate(Bm):
        Um = torch.zeros_like(Bm)
        for _ in range(3):
            mg.solve(Um, Bm, rtol=1e-10, max_iters=60, use_initial_guess=False)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        reps = [mg.solve(Um, Bm, rtol=1e-10, max_iters=60, use_initial_guess=False)[1] for _ in range(steps)]
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / steps
        nr = 1 if Bm.dim() == 1 else Bm.shape[0]
        return Um, reps[-1], t, nr

    U, rep, t1, _ = rate(b)
    B32 = torch.tensor(np.stack([dec.meshes.uniform(1 + j, n) for j in range(NRHS)]), device="cuda")
    _, rep32, t32, _ = rate(B32)
    res = {"vertices": n, "cycle": "V(3,3) Chebyshev-Jacobi [λ/4, λ], dense FP64 solve on L0 (12 vertices)",
           "refinement_steps": int(rep.iterations), "v_cycles": int(rep.iterations),
           "max_rel_residual": rep.max_rel_residual, "converged": bool(rep.converged),
           "ms_per_solve_1rhs": 1e3 * t1, "solves_per_s_1rhs": 1.0 / t1,
           "solves_per_s_32rhs": NRHS / t32, "ms_per_32rhs": 1e3 * t32,
           "bytes_per_solve_1rhs": mg.solve_traffic(1, int(rep.iterations))}
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        oracle, O, md = oracle_hierarchy(6, threads)
        bh = b.cpu().numpy()
        ue, rel, cyc, lmax = oracle.fp64_solve(md, bh, rtol=1e-13)
        u = U.cpu().numpy()
        res["rel_error_vs_fp64_oracle_solve"] = float(np.linalg.norm(u - ue) / np.linalg.norm(ue))
        res["oracle_solve"] = f"{cyc} oracle V(3,3) cycles to {rel:.1e}"
        # the same V-cycle on the host cores (the oracle), to 1e-10
        import scipy.sparse as sp
        cp, rv, nz, shape = md.op(0)
        A = sp.csc_matrix((nz, rv, cp), shape=shape).tocsr()
        t0 = time.perf_counter()
        uc, c = np.zeros(n), 0
        while c < 40:
            uc = O.plain_vcycles(md, uc, bh, 1, 1, 3, 3, 0.8, 4.0, lmax)
            c += 1
            if np.linalg.norm(bh - A @ uc) / np.linalg.norm(bh) <= 1e-10:
                break
        tc = time.perf_counter() - t0
        res["cpu_same_cycle"] = {"seconds_per_solve": tc, "v_cycles": c, "threads": threads,
                                 "kind": "port (oracle V(3,3) FP64, residual checks included)"}
    del mg
    torch.cuda.empty_cache()
    return res


def measure_config3(dec, args, common):
    """Mixed precision at L8 to 1e-10: 32 right-hand sides (seeds 2..33), FP32 V-cycles (the
    headline cycle) inside FP64 iterative refinement; errors against the oracle's FP64-only solve
    (to 1e-13 on the host, for the first `args.oracle_rhs` right-hand sides)."""
    import torch
    ico = dec.meshes.icosahedron()
    mg = dec.MultigridData(ico, LEVEL, precision=1, **common)
    if args.rhs_block == 0:
        mg.autotune(NRHS, reps=2)
    n = mg.n
    B = torch.tensor(np.stack([dec.meshes.uniform(s, n) for s in range(2, 2 + NRHS)]), device="cuda")
    U = torch.zeros_like(B)
    steps = max(1, args.steps)
    for _ in range(max(1, args.warmup)):
        mg.solve(U, B, rtol=1e-10, max_iters=60, use_initial_guess=False)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    reps = [mg.solve(U, B, rtol=1e-10, max_iters=60, use_initial_guess=False)[1] for _ in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / steps
    rep = reps[-1]
    res = {"rtol": 1e-10, "solves_per_s": NRHS / t, "ms_per_32rhs": 1e3 * t,
           "refinement_steps": int(rep.iterations), "v_cycles": int(rep.iterations) * common["inner_cycles"],
           "converged": bool(rep.converged), "max_rel_residual": rep.max_rel_residual,
           "bytes_per_step": mg.solve_traffic(NRHS, int(rep.iterations))}
    if not args.no_cpu and args.oracle_rhs > 0:
        threads = os.cpu_count() or 1
        oracle, O, md = oracle_hierarchy(LEVEL, threads)
        lmax = [oracle.level_lmax(md, l) for l in range(md.nlevels)]
        Bh, Uh = B.cpu().numpy(), U.cpu().numpy()
        errs, t0 = [], time.perf_counter()
        for j in range(min(NRHS, args.oracle_rhs)):
            ue, rel, _, _ = oracle.fp64_solve(md, Bh[j], rtol=1e-13, lmax=lmax)
            errs.append(float(np.linalg.norm(Uh[j] - ue) / np.linalg.norm(ue)))
        res["max_rel_error_vs_fp64_oracle_solve"] = max(errs)
        res["oracle_rhs_checked"] = len(errs)
        res["oracle_seconds"] = time.perf_counter() - t0
    del mg, B, U
    torch.cuda.empty_cache()
    return res


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------------------------------
# Ranks: one process per GPU, each solving its own right-hand sides (replicas, no data-path
# collective); the process group carries only the barrier and the max-over-ranks timing.
# ------------------------------------------------------------------------------------------
def init_dist(world, backend="nccl", timeout_s=300):
    """The process group of a world > 1 run (rendezvous from MASTER_ADDR / MASTER_PORT), with a
    short timeout so that ranks waiting on a dead one end with an error."""
    if world <= 1:
        return
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def rank_seeds(rank, nrhs=NRHS):
    """The right-hand-side seeds of a rank: rank r solves seeds 2 + r·nrhs .. 1 + (r+1)·nrhs."""
    return [2 + j + nrhs * rank for j in range(nrhs)]


def collectives(world, device):
    """(barrier, max_over_ranks) for a world of `world` ranks; max_over_ranks reduces a float on
    `device` ("cuda" under NCCL, "cpu" under gloo).  Identity functions for one rank."""
    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world > 1:
            import torch
            import torch.distributed as dist
            t = torch.tensor([x], dtype=torch.float64, device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    return barrier, max_over_ranks


def whole_job_rate(nrhs, world, steps, seconds):
    """Solves per second of the whole job: every rank's right-hand sides over the slowest rank's
    time (seconds is already the max over ranks)."""
    return nrhs * world * steps / seconds


# ------------------------------------------------------------------------------------------
# CPU baseline (the oracle, on the host cores)
# ------------------------------------------------------------------------------------------
def cpu_reference_solve(O, md, A, b, budget_s=30.0):
    """One reference-algorithm solve (Multigrid.jl V-cycles, Krylov CG smoother with 3 steps,
    FP64) until ‖b - A u‖/‖b‖ ≤ RTOL or the time budget runs out.  Returns (seconds, cycles,
    residual, converged)."""
    u = np.zeros_like(b)
    nb = np.linalg.norm(b)
    t0 = time.perf_counter()
    cycles = 0
    rel = 1.0
    while True:
        u = O.mu_cycles(md, u, b, 1, 1)
        cycles += 1
        rel = np.linalg.norm(b - A @ u) / nb
        if rel <= RTOL or time.perf_counter() - t0 > budget_s or cycles >= 50:
            break
    return time.perf_counter() - t0, cycles, float(rel), bool(rel <= RTOL)


def build_cpu_reference(threads):
    sys.path.insert(0, str(ROOT))
    import oracle
    import scipy.sparse as sp
    O = oracle.load()
    O.set_num_threads(threads)
    ico = O.icosahedron()
    md = O.build_mg(ico, LEVEL, O.CIRCUMCENTER, SHIFT, 1.0, 3)
    cp, rv, nz, shape = md.op(0)
    A = sp.csc_matrix((nz, rv, cp), shape=shape).tocsr()
    return O, md, A


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    dec = load_package()
    O, md, A = build_cpu_reference(threads)
    n = A.shape[0]
    for w in range(args.warmup):
        cpu_reference_solve(O, md, A, dec.meshes.uniform(2 + w, n), budget_s=20.0)
    times, cycles, conv = [], [], True
    for s in range(args.steps):
        t, c, rel, ok = cpu_reference_solve(O, md, A, dec.meshes.uniform(2 + s % NRHS, n), budget_s=30.0)
        times.append(t)
        cycles.append(c)
        conv = conv and ok
    total = sum(times)
    value = args.steps / total
    line = {
        "impl": "reference", "metric": "icosphere-L8 Helmholtz solves/s to 1e-8 relative residual",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "icosphere L8 (655,362 vertices) Helmholtz (L + I) u = b, b uniform[-1,1], "
                               "to 1e-8 relative residual; one right-hand side per step",
                   "algorithm": "Multigrid.jl V-cycles, Krylov CG smoother (3 steps), CG on the coarsest "
                                "level, FP64 (the reference's multigrid_vcycles)",
                   "converged": conv, "cycles_per_solve": cycles},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} single-RHS solves of the L8 workload on {threads} host threads "
                                   "(CPU oracle restating the reference algorithm; Julia is not installed)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    init_dist(world, "nccl")
    dec = load_package()
    ico = dec.meshes.icosahedron()
    t_setup = time.perf_counter()
    common = dict(shift=SHIFT, center="circumcenter", project_radius=1.0, smoother=1, pre=args.pre,
                  post=args.post, cheb_ratio=args.cheb_ratio, rhs_block=args.rhs_block,
                  inner_cycles=args.inner_cycles, coarse_max=args.coarse_max)
    # a profiling run drives the refinement loop from the host, so that every kernel is a graph
    # node the profiler follows (kernels inside the device loop's conditional node are not)
    mg = dec.MultigridData(ico, LEVEL, precision=1, **dict(common, device_loop=0 if args.profile else 1))
    mg64 = dec.MultigridData(ico, LEVEL, precision=0, **common)
    setup_s = time.perf_counter() - t_setup
    n = mg.level_info(0)[0]
    seeds = rank_seeds(rank)
    B = torch.tensor(np.stack([dec.meshes.uniform(s, n) for s in seeds]), device="cuda")
    U = torch.zeros_like(B)
    tuned = mg.autotune(NRHS, reps=3) if args.rhs_block == 0 else args.rhs_block
    if args.rhs_block == 0:
        mg64.autotune(NRHS, reps=3)
    stream = torch.cuda.current_stream()

    barrier, max_over_ranks = collectives(world, "cuda")

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps = [fn() for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3), reps

    # --- headline: mixed-precision solve, inputs resident in HBM ---
    def solve32():
        return mg.solve(U, B, rtol=RTOL, max_iters=100, use_initial_guess=False)[1]

    sampler = ClockSampler(local)
    for _ in range(args.warmup):
        solve32()
    barrier()
    torch.cuda.synchronize()

    def load_for(seconds):  # the same solves, untimed, so the sampler sees the GPU under this load
        t_end = time.perf_counter() + seconds
        while time.perf_counter() < t_end:
            solve32()
        torch.cuda.synchronize()

    sampler.start()
    load_for(0.6)
    torch.cuda.nvtx.range_push("timed")
    t_ours, reps = timed(solve32, args.steps, 0)
    torch.cuda.nvtx.range_pop()
    load_for(0.6)
    clocks = sampler.stop()
    clocks["window"] = "0.6 s of the same solves before and after the timed region, and the timed region"
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "solves_per_s": whole_job_rate(NRHS, world, args.steps, t_ours),
                              "v_cycles": int(reps[-1].iterations), "rhs_block": int(tuned)}), flush=True)
        return
    rep0 = reps[-1]
    converged = all(r.converged for r in reps)
    value = whole_job_rate(NRHS, world, args.steps, t_ours)
    launches = int(sum(r.launches for r in reps))

    # --- error against an FP64-only solve (GPU, FP64 V-cycles to 1e-12) ---
    U64 = torch.zeros_like(B)
    mg64.solve(U64, B, rtol=1e-12, max_iters=200)
    err = float(((U - U64).norm(dim=1) / U64.norm(dim=1)).max())

    # --- plain FP64 V-cycle solves of the same workload (the comparison method): the same cycle
    # options and the other configurations measured best for the FP32 path, the fastest counted ---
    cheb64 = []
    for cfg in ({}, dict(pre=3, post=3, cheb_ratio=4.0, inner_cycles=3), dict(pre=1, post=2, cheb_ratio=4.0,
                                                                              inner_cycles=2)):
        m64 = mg64 if not cfg else dec.MultigridData(ico, LEVEL, precision=0, **dict(common, **cfg))
        if cfg and args.rhs_block == 0:
            m64.autotune(NRHS, reps=2)

        def solve64():
            return m64.solve(U64, B, rtol=RTOL, max_iters=100, use_initial_guess=False)[1]

        t_plain, reps64 = timed(solve64, max(1, args.steps), 1)
        o = m64.options
        cheb64.append({"cycle": f"V({o.pre},{o.post}) ratio {o.cheb_ratio:g}, {o.inner_cycles} per step",
                       "solves_per_s": whole_job_rate(NRHS, world, max(1, args.steps), t_plain),
                       "refinement_steps": int(reps64[-1].iterations)})
        if cfg:
            del m64
    torch.cuda.empty_cache()
    best64 = max(cheb64, key=lambda r: r["solves_per_s"])
    cheb64_value = best64["solves_per_s"]

    # --- the reference algorithm's V-cycle in FP64 (Krylov CG smoother, 3 steps before and after,
    # Multigrid.jl:814-872) on the same workload; the plain baseline is the faster of the two ---
    mgcg = dec.MultigridData(ico, LEVEL, precision=0, smoother=2, pre=3, post=3, shift=SHIFT,
                             center="circumcenter", project_radius=1.0, coarse_max=args.coarse_max,
                             inner_cycles=args.inner_cycles, rhs_block=args.rhs_block)
    if args.rhs_block == 0:
        mgcg.autotune(NRHS, reps=2)
    Ucg = torch.zeros_like(B)

    def solve_cg():
        return mgcg.solve(Ucg, B, rtol=RTOL, max_iters=100, use_initial_guess=False)[1]

    t_cg, reps_cg = timed(solve_cg, max(1, args.steps), 1)
    cg64_value = whole_job_rate(NRHS, world, max(1, args.steps), t_cg)
    assert reps_cg[-1].converged == 1
    del mgcg, Ucg
    torch.cuda.empty_cache()
    plain_value = max(cheb64_value, cg64_value)

    # --- e2e through the C ABI with host buffers: every step copies its b (pinned host FP64) in
    # and its u out, submitted through the pipelined host-buffer solve (three steps in flight, so
    # the neighbouring steps' copies overlap each step's compute) ---
    Bh = B.cpu().pin_memory()
    Uh = [torch.zeros_like(Bh).pin_memory() for _ in range(3)]

    def solve_host_steps(count):
        pending, reps = [], []
        for i in range(count):
            if len(pending) == 3:
                reps.append(pending.pop(0).wait()[1])
            pending.append(mg.solve_host_submit(Uh[i % 3], Bh, rtol=RTOL, max_iters=100, use_initial_guess=False))
        reps += [p.wait()[1] for p in pending]
        return reps

    solve_host_steps(max(args.warmup, 1))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_reps = solve_host_steps(args.steps)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    assert all(r.converged == 1 for r in e2e_reps)
    e2e_value = whole_job_rate(NRHS, world, args.steps, t_e2e)
    bytes_vec = NRHS * n * 8

    # --- roofline of the dominant kernel, timed alone: the first Chebyshev step after the fused
    # prolongation on the finest level (k_sweep_ap, the largest share of the solve's launch list);
    # beside it the plain Chebyshev step (k_sweep) ---
    ms, algo_bytes = mg.time_kernel(6, 0, NRHS, reps=20)
    ms_sw, bytes_sw = mg.time_kernel(0, 0, NRHS, reps=20)
    peak, peak_kind = measured_peaks()
    achieved = algo_bytes / (ms * 1e-3) / 1e9
    traffic = traffic_per_launch("k_sweep_ap")

    # --- the whole step's algorithmic bytes (every kernel of the solve graph) against its time ---
    step_bytes = mg.solve_traffic(NRHS, int(rep0.iterations))
    step_gbs = step_bytes / (t_ours / args.steps) / 1e9

    # --- config 2 (L6 FP64 to 1e-10) and config 3 (L8 mixed precision to 1e-10) ---
    config2 = measure_config2(dec, args) if (rank == 0 and not args.no_configs) else None
    config3 = measure_config3(dec, args, common) if (rank == 0 and not args.no_configs) else None

    # --- batched uneven workload (512 solves over 8 meshes, one graph per step) ---
    batched = measure_batched(dec, args) if (rank == 0 and not args.no_batch) else None

    # --- learned smoother (trained here), L8 and L9 ---
    learned_res = measure_learned(dec, args, B, U64, common, timed) if args.train_steps > 0 else None

    # --- DEC operator kernels (wedges, d, star, Laplacian) at full size ---
    operators = measure_operators(dec, peak, cpu=not args.no_cpu) if (rank == 0 and not args.no_ops) else None

    # --- CPU baseline (rank 0, N = 1 only): the reference algorithm on the host cores ---
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        O, md, A = build_cpu_reference(threads)
        t, c, rel, ok = cpu_reference_solve(O, md, A, dec.meshes.uniform(2, n), budget_s=30.0)
        cpu = {"value": 1.0 / t, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"1 right-hand side (seed 2) of the L8 workload: {c} reference V-cycles "
                         f"(Krylov CG smoother, FP64) to {rel:.2e} in {t:.2f} s on {threads} host threads"}

    learned_ratio = None
    if learned_res:
        cands = [(k, c, r) for k in ("L8_learned_fp32", "L8_learned_fp32_mma_sync") for c, r in learned_res[k].items()
                 if r["converged"]]
        if cands:
            k, c, r = max(cands, key=lambda x: x[2]["solves_per_s"])
            learned_ratio = {"value": r["solves_per_s"] / plain_value, "learned_solves_per_s": r["solves_per_s"],
                             "plain_fp64_solves_per_s": plain_value, "learned_cycle": f"{k} {c}",
                             "fallback_iteration": r["fallback_iteration"], "target": 3.0}
    if rank == 0:
        line = {
            "metric": "icosphere-L8 Helmholtz solves/s to 1e-8 relative residual",
            "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_ours / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle in f64 refinement",
            "data": "synthetic",
            "config": {
                "workload": "icosphere L8 (655,362 vertices, 1,310,720 triangles) Helmholtz (L + I) u = b, "
                            f"{NRHS} RHS per GPU per step (seeds 2..33), to 1e-8 relative residual",
                "method": f"FP32 Chebyshev-Jacobi V({args.pre},{args.post})-cycles (interval [λ/{args.cheb_ratio:g}, λ]), "
                          f"{args.inner_cycles} per "
                          "FP64 iterative-refinement step, dense FP64 solve on the coarsest level used "
                          f"(coarse_max {args.coarse_max}), locality-ordered levels",
                "rhs_panel_width": int(tuned), "refinement_steps": int(rep0.iterations),
                "v_cycles_per_solve": int(rep0.iterations) * args.inner_cycles,
                "converged": converged, "max_rel_residual": rep0.max_rel_residual,
                "max_rel_error_vs_fp64_solve": err,
                "l2": "inputs larger than L2 (b: 168 MB FP64 per step)",
                "parallelism": f"replicas x{world} (independent batches, no collective)",
                "setup_seconds": setup_s,
                "tuned_variants": {k: v for k, v in dec.tune_entries().items() if k.startswith(("sweep/", "cheb2/"))},
            },
            "learned_fp32_vs_plain_fp64": learned_ratio,
            "comparison": {"plain_fp64_vcycle_solves_per_s": plain_value,
                           "speedup_vs_plain_fp64": value / plain_value,
                           "plain_fp64_chebyshev": best64,
                           "plain_fp64_chebyshev_configs": cheb64,
                           "plain_fp64_reference_cg_smoother": {"solves_per_s": cg64_value,
                                                                "refinement_steps": int(reps_cg[-1].iterations)},
                           "plain": "the faster of the two FP64 V-cycle solves"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": f"k_sweep_ap<float,{int(tuned)}> finest level (first step after the prolongation)",
                         "algorithmic_bytes_per_launch": algo_bytes, "ms_per_launch": ms,
                         "peak_kind": f"{peak_kind} (HBM copy, burst)",
                         "plain_step": {"kernel": f"k_sweep<float,{int(tuned)},6> finest level (middle Chebyshev step)",
                                        "ms_per_launch": ms_sw, "algorithmic_bytes_per_launch": bytes_sw,
                                        "achieved": bytes_sw / (ms_sw * 1e-3) / 1e9,
                                        "frac": bytes_sw / (ms_sw * 1e-3) / 1e9 / peak,
                                        "traffic": traffic_per_launch("k_sweep")},
                         "step_algorithmic_bytes": step_bytes, "step_GB/s": step_gbs,
                         "step_frac": step_gbs / peak},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": bytes_vec,
                    "d2h_bytes_per_step": bytes_vec,
                    "api": "MultigridData.solve_host_submit / wait (dec_mg_solve_host_submit / _wait): "
                           "pinned host b in, host u out, three steps in flight"},
            "gpu_launches": launches,
            "clocks": clocks,
            "operators": operators,
            "learned_smoother": learned_res,
            "config2_L6_fp64": config2,
            "config3_L8_mixed_1e-10": config3,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_op(args):
    """One DEC operator kernel alone on icosphere L`mesh_level` (circumcentric duals), `steps`
    back-to-back applications after `warmup`, FP64 or FP32 (--dtype): the entry point for ncu
    captures of the operator kernels."""
    import torch
    dec = load_package()
    m = dec.meshes.icosphere(args.mesh_level)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                 center="circumcenter")
    tdt = torch.float64 if args.dtype == "float64" else torch.float32
    f = torch.rand(g.nv, dtype=tdt, device="cuda")
    a = torch.rand(g.ne, dtype=tdt, device="cuda")
    b = torch.rand(g.ne, dtype=tdt, device="cuda")
    t = torch.rand(g.nt, dtype=tdt, device="cuda")
    ops = {
        "laplacian": (dec.laplace_beltrami(g, args.dtype), f),
        "d0": (dec.dec_differential(0, g, args.dtype), f),
        "d1": (dec.dec_differential(1, g, args.dtype), a),
        "star1_geometric": (dec.hodge_operator(1, g, dtype=args.dtype, hodge="geometric"), a),
    }
    wedges = {"wedge01": (dec.dec_wedge_product(0, 1, g, args.dtype), f, a),
              "wedge11": (dec.dec_wedge_product(1, 1, g, args.dtype), a, b),
              "wedge02": (dec.dec_wedge_product(0, 2, g, args.dtype), f, t)}
    variant = None
    if args.op == "wedge11_batched":
        # `count` FP32 pairs in one batched launch, pairs per thread from --variant or the autotuner
        w = dec.dec_wedge_product(1, 1, g, "float32")
        A = torch.rand((args.count, g.ne), dtype=torch.float32, device="cuda")
        B = torch.rand((args.count, g.ne), dtype=torch.float32, device="cuda")
        y = torch.empty((args.count, g.nt), dtype=torch.float32, device="cuda")
        key = f"w11pairs/f32/n{int(np.log2(g.nt))}"
        if args.variant:
            dec.tune_set(key, args.variant)
        else:
            w.autotune(args.count, reps=3)
        variant = {key: dec.tune_get(key)}
        fn = lambda: w.batched(A, B, y)
    elif args.op in ops:
        op, x = ops[args.op]
        y = torch.empty(op.shape[0], dtype=tdt, device="cuda")
        if args.op == "laplacian":
            key = f"ell/{'f64' if args.dtype == 'float64' else 'f32'}/W7/n{int(np.log2(g.nv))}"
            if args.variant:
                dec.tune_set(key, args.variant)
            elif args.autotune:
                op.autotune(reps=10)
            variant = {key: dec.tune_get(key)}
        fn = lambda: op.apply(x, y)
    else:
        w, x1, x2 = wedges[args.op]
        y = torch.empty(w.len_out, dtype=tdt, device="cuda")
        fn = lambda: w(x1, x2, y)
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    us = 1e3 * e0.elapsed_time(e1) / args.steps
    rec = {"op": args.op, "dtype": "float32" if args.op == "wedge11_batched" else args.dtype,
           "mesh_level": args.mesh_level, "nv": g.nv, "ne": g.ne, "nt": g.nt,
           "us_per_launch": us, "variant": variant}
    if args.op == "wedge11_batched":
        by = args.count * (2.0 * g.ne * 4 + g.nt * 4) + g.nt * (12 + 3 * 4)
        rec.update({"count": args.count, "bytes": by, "GB/s": by / us / 1e3})
    print(json.dumps(rec), flush=True)


def run_kernel(args):
    """One V-cycle kernel alone (dec_mg_time_kernel) on icosphere L`mesh_level` with NRHS
    right-hand sides: the entry point for ncu captures of a single kernel."""
    import torch
    dec = load_package()
    kinds = {"sweep": 0, "residual": 1, "restrict": 2, "prolong": 3, "mlp": 4, "pair": 5, "sweep_p0": 6,
             "sweep_p1": 7}
    kind = kinds[args.kernel]
    mg = dec.MultigridData(dec.meshes.icosahedron(), args.mesh_level, shift=SHIFT, center="circumcenter",
                           project_radius=1.0, smoother=3 if kind == 4 else 1, pre=max(1, args.pre),
                           post=max(1, args.post),
                           precision=args.precision, rhs_block=32, coarse_max=args.coarse_max)
    if kind == 5 and args.variant:  # patch rows of the pair
        n = mg.level_info(0)[0]
        dec.tune_set(f"cheb2/f32/K32/W6/n{int(np.log2(n))}", args.variant)
    if kind == 4:
        mlp = dec.SmootherMLP(4)
        mlp.set_engine(args.mlp_engine)
        mg.set_smoother_mlp(mlp)
    for _ in range(args.warmup):
        mg.time_kernel(kind, 0, NRHS, reps=1)
    ms, by = mg.time_kernel(kind, 0, NRHS, reps=args.steps)
    torch.cuda.synchronize()
    nv = mg.level_info(0)[0]
    line = {"kernel": args.kernel, "mesh_level": args.mesh_level, "precision": args.precision, "nrhs": NRHS,
            "ms_per_launch": ms,
            "algorithmic_bytes": by, "GB/s": by / (ms * 1e-3) / 1e9}
    if kind == 4:
        line["tensor_TFLOP/s"] = 10240.0 * nv * NRHS / (ms * 1e-3) / 1e12
        line["mlp_engine"] = args.mlp_engine
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pre", type=int, default=0, help="Chebyshev steps before the coarse correction")
    ap.add_argument("--post", type=int, default=2, help="Chebyshev steps after it")
    ap.add_argument("--sweeps", type=int, default=None, help="sets --pre and --post")
    ap.add_argument("--cheb-ratio", type=float, default=3.0, dest="cheb_ratio",
                    help="Chebyshev interval [λmax / ratio, λmax]")
    ap.add_argument("--inner-cycles", type=int, default=3, dest="inner_cycles")
    ap.add_argument("--coarse-max", type=int, default=170, dest="coarse_max")
    ap.add_argument("--rhs-block", type=int, default=0, dest="rhs_block")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ops", action="store_true", help="skip the operator-kernel roofline section")
    ap.add_argument("--profile", action="store_true",
                    help="run only the timed mixed-precision solves (inside an NVTX range 'timed')")
    ap.add_argument("--kernel", choices=["sweep", "residual", "restrict", "prolong", "mlp", "pair", "sweep_p0",
                                         "sweep_p1"],
                    help="time one V-cycle kernel alone (steps launches after warmup) and exit")
    ap.add_argument("--mesh-level", type=int, default=LEVEL, dest="mesh_level")
    ap.add_argument("--precision", type=int, default=1, choices=[1, 2],
                    help="V-cycle storage for --kernel: 1 FP32, 2 FP16 (FP32 arithmetic)")
    ap.add_argument("--op", choices=["laplacian", "d0", "d1", "star1_geometric", "wedge01", "wedge11", "wedge02",
                                     "wedge11_batched"],
                    help="time one DEC operator kernel alone (steps launches after warmup) and exit")
    ap.add_argument("--dtype", default="float64", choices=["float64", "float32"])
    ap.add_argument("--count", type=int, default=64, help="--op wedge11_batched: form pairs per launch")
    ap.add_argument("--autotune", action="store_true", help="--op laplacian: autotune the apply's variant first")
    ap.add_argument("--variant", type=int, default=0,
                    help="--op laplacian: rows per thread (1, 2, 4); --kernel pair: patch rows (128, 256, 512)")
    ap.add_argument("--no-batch", action="store_true", dest="no_batch", help="skip the batched-workload section")
    ap.add_argument("--no-configs", action="store_true", dest="no_configs",
                    help="skip the L6 FP64 and L8 1e-10 sections")
    ap.add_argument("--oracle-rhs", type=int, default=8, dest="oracle_rhs",
                    help="right-hand sides of the L8 1e-10 section whose error is checked against the oracle's "
                         "FP64 solve on the host")
    ap.add_argument("--mlp-engine", default="tcgen05", choices=["mma", "tcgen05"], dest="mlp_engine",
                    help="kernel engine of the learned smoothing step for --kernel mlp")
    ap.add_argument("--train", action="store_true", help="train the learned smoother alone (--train-steps) and exit")
    ap.add_argument("--train-steps", type=int, default=20000, dest="train_steps",
                    help="Adam steps of the learned smoother (0 skips the learned-smoother section)")
    args = ap.parse_args()
    if args.sweeps is not None:
        args.pre = args.post = args.sweeps
    if args.train:
        run_train(args)
    elif args.op:
        run_op(args)
    elif args.kernel:
        run_kernel(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
