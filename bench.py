"""Benchmark: ligands docked per second on the batched uneven search workload.

Workload (one step): 256 synthetic ligands (10-60 heavy atoms, 0-15 rotatable bonds, seeds 0-255 on rank 0)
docked against the 1,500-atom synthetic receptor (22.5 A box, 61^3 x 8 Vina maps, FP32) with 32 MC chains x
2,000 MC steps each (BFGS local optimisation, Vina iteration rule), BFGS refinement, exact polish of the top 32
chains and finalize (top 9 poses). Ranks shard ligands (rank r docks seeds 256r .. 256r+255); no collective on
the data path (weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). ``value`` times the search on device-resident inputs (maps, packed ligands);
``e2e`` times the public ``dock_screen`` call from host arrays (map build, packing, host<->device copies,
search, results back on the host). ``--impl reference`` times the reference's own search, unmodified (its driver
``search.dock_problem_kernel`` with device "cpu" and its g++/OpenMP kernels, installed under baseline/_ref), on the
host cores, on a 4-ligand sample.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_LIGANDS = 256
CHAINS = 32
MC_STEPS = 2000
METRIC = "ligands docked/s (plain FP32 search: 32 MC chains x 2000 steps + BFGS, top-9 poses)"
UNIT = "ligands/s"
WORKLOAD = ("batched uneven search: 256 synthetic ligands (10-60 heavy atoms, 0-15 torsions) x 32 chains x 2000 "
            "MC steps vs 1500-atom receptor, 61^3 x 8 Vina maps (FP32)")


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ligands", type=int, default=N_LIGANDS)
    ap.add_argument("--mc-steps", type=int, default=MC_STEPS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mc-variant", type=int, default=0,
                    help="MC launch variant (1-3: 4, 6 or 8 resident blocks per SM); 0 = the autotuner's choice")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the map-builder / map-precision section")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-proposal section (FP16 maps + learned proposal vs plain FP32 at equal "
                         "median gap, screening shapes, reduced ligand counts)")
    ap.add_argument("--learned-train", type=int, default=512, help="training ligands of the learned-proposal section")
    ap.add_argument("--learned-eval", type=int, default=256, help="held-out ligands of the learned-proposal section")
    ap.add_argument("--ab", action="store_true", help="learned proposal vs plain MC at equal step budget")
    ap.add_argument("--ab-train", type=int, default=256, help="fresh ligands for the proposal's training data")
    ap.add_argument("--ab-eval", type=int, default=256, help="held-out ligands for the A/B comparison")
    ap.add_argument("--ab-variants", default="learned_f16:32:0.3",
                    help="learned variants name:segment_steps:learned_fraction[:chain|ligand|dagger training[:tries"
                         "[:hint[:n_comp]]]], comma separated (hint: the network reads the ligand-best hint; n_comp 3: "
                         "translation mixture)")
    ap.add_argument("--screen", action="store_true",
                    help="screening comparison on the 8,000-atom receptor with 8-80-atom ligands (FP16 + learned "
                         "proposal vs plain FP32 at equal median gap)")
    ap.add_argument("--screen-train", type=int, default=1536, help="fresh ligands for the screening proposal's training")
    ap.add_argument("--screen-eval", type=int, default=1024, help="held-out ligands of the screening comparison")
    ap.add_argument("--screen-log-cap", type=int, default=4_000_000, help="training moves kept per collection")
    ap.add_argument("--screen-variants", default="learned_dagger2:32:0.6>0.3@64:dagger2:4:0:3",
                    help="learned variants of the screening comparison (as --ab-variants; dagger, dagger2, ...: "
                         "that many self-training rounds)")
    ap.add_argument("--screen-full", action="store_true",
                    help="the full-form screening run in place of the bench line: --screen-full-ligands ligands on "
                         "the 8,000-atom receptor docked in one batch by the learned FP16 search and by the plain FP32 "
                         "search, gaps on a subset, the reference's CPU search on a sample")
    ap.add_argument("--screen-full-ligands", type=int, default=16384)
    ap.add_argument("--screen-full-learned-steps", default="400,600",
                    help="budgets of the learned search (comma separated), interpolated to the plain run's gap")
    ap.add_argument("--screen-full-plain-steps", type=int, default=3000)
    ap.add_argument("--screen-full-subset", type=int, default=1024, help="ligands whose gap is measured")
    ap.add_argument("--screen-full-cpu", type=int, default=16,
                    help="ligands of the first 256 timed with the reference's CPU search (0: none)")
    return ap.parse_args()


def _workload(rank, n_lig, mc_steps):
    from adock_b200 import params, synth
    rec = synth.config_receptor(0)
    ligs = synth.ligand_set(n_lig, (10, 60), (0, 15), seed0=rank * n_lig)
    cfg = params.workload_preset(CHAINS, mc_steps)
    return rec, ligs, cfg


def _cpu_sample(ligs):
    """4 ligands at the 1/8, 3/8, 5/8, 7/8 quantiles of the heavy-atom count (a size-representative sample)."""
    order = sorted(range(len(ligs)), key=lambda i: (ligs[i].n, i))
    pick = [order[int(len(order) * f)] for f in (0.125, 0.375, 0.625, 0.875)]
    return [ligs[i] for i in pick]


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.rows, self.proc = [], None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(gpu_index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            p = [x.strip() for x in line.split(",")]
            if len(p) == 7:
                self.rows.append(p)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except ValueError:
                continue
            for n, v in zip(names, r[3:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        load = [s for s in sm if mx and s > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_figure(name):
    """A per-evaluation figure of the MC kernel from the committed ncu summary (None if absent):
    dram_bytes_per_atom_eval, warp_instructions_per_eval."""
    f = ROOT / "profiles" / "mc_kernel_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(name + ":"):
            return float(line.split(":")[1])
    return None


def _traffic_per_atom_eval():
    return _profile_figure("dram_bytes_per_atom_eval")


REF_INSTALL = ROOT / "baseline" / "_ref"


def _stock_reference():
    """The reference package installed unmodified under baseline/_ref (pip install --target), imported
    with empty stand-ins for cupy and rdkit, which its CPU path does not use. Its CPU kernels are compiled on first
    use by its own adock.cpukernel (g++ -O3 -march=native -ffast-math -fopenmp, all host threads) into a temporary
    cache. Returns the modules, or None when the install is absent."""
    if not (REF_INSTALL / "adock" / "search.py").exists():
        return None
    import tempfile
    import types
    for name in ("cupy", "rdkit", "rdkit.Chem"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["rdkit"].Chem = sys.modules["rdkit.Chem"]
    os.environ.setdefault("ADOCK_CPU_CACHE", tempfile.mkdtemp(prefix="adock_ref_cpu_"))
    os.environ.setdefault("ADOCK_CPU_THREADS", str(len(os.sched_getaffinity(0))))
    if str(REF_INSTALL) not in sys.path:
        sys.path.insert(0, str(REF_INSTALL))
    from adock import grid, ligand, scoring, search
    return types.SimpleNamespace(grid=grid, ligand=ligand, scoring=scoring, search=search,
                                 threads=int(os.environ["ADOCK_CPU_THREADS"]))


def _reference_problem(A, rec, ligs):
    """The reference's Problem for a ligand list: its make_gridset (its CPU grid kernel), LigandBatch, Problem and
    receptor padding, unchanged; built once per sample, outside the timed searches (its screening caller shares one
    map set across all ligands, screen.py:55-56)."""
    import numpy as np
    import torch
    from adock_b200 import params
    sfp = params.sf_params("vina")          # the same constants as the reference's config/adock.json "scoring"
    lt = np.unique(np.concatenate([[0]] + [l.types for l in ligs]))
    gs = A.grid.make_gridset([rec], sfp, params.GRID_SPACING, params.OUT_OF_BOX_PENALTY, device="cpu", lig_types=[lt])
    prob = A.search.Problem(gs, A.ligand.LigandBatch(ligs, "cpu"), torch.zeros(len(ligs), dtype=torch.long),
                            A.scoring.PairPotential(sfp), rec=A.search.pad_receptors([rec], "cpu"))
    prob._box = (torch.tensor(rec["center"], dtype=torch.float32)[None].expand(len(ligs), 3), [rec["size"]] * len(ligs))
    return prob


def _reference_search(A, prob, cfg, seed=0):
    """One stock reference search (dock_problem_kernel with device "cpu") on the host cores: (seconds, results)."""
    t0 = time.perf_counter()
    res = A.search.dock_problem_kernel(prob, *prob._box, cfg, seed=seed)
    return time.perf_counter() - t0, res


def run_reference(args, rank, world):
    """Reference arm: the reference's own search (its driver, Stage A, CPU kernels, finalize; unmodified) on the host
    cores, one 4-ligand sample of the workload per step."""
    if rank != 0:
        return None
    import torch
    A = _stock_reference()
    if A is None:
        return {"impl": "reference", "unavailable": "the reference package is not installed under baseline/_ref"}
    torch.set_num_threads(A.threads)
    rec, ligs, cfg = _workload(0, args.ligands, args.mc_steps)
    sample = _cpu_sample(ligs)
    prob = _reference_problem(A, rec, sample)
    for _ in range(args.warmup):      # compiles the reference's kernels, pages in the inputs (20-step budget, untimed)
        _reference_search(A, prob, dict(cfg, mc_steps=20, mc_segment=20))
    times = [_reference_search(A, prob, cfg)[0] for _ in range(args.steps)]
    v = len(sample) * len(times) / sum(times)
    sample_desc = (f"{len(sample)} ligands of the workload (heavy atoms {[p.n for p in sample]}) x {CHAINS} chains x "
                   f"{args.mc_steps} steps, the full stock search per step (maps built once, untimed)")
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": WORKLOAD, "ligands_per_step": len(sample), "chains": CHAINS, "mc_steps": args.mc_steps,
                       "parallelism": "host cores (OpenMP)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": A.threads, "kind": "reference", "sample": sample_desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    from adock_b200 import _lib, params
    from adock_b200.grid import make_gridset
    from adock_b200.kernel import B200KernelProblem
    from adock_b200.ligand import LigandBatch
    from adock_b200.problem import PairPotential, Problem, pad_receptors
    from adock_b200.screen import dock_screen
    from adock_b200.search import dock_problem_kernel

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rec, ligs, cfg = _workload(rank, args.ligands, args.mc_steps)
    sfp = params.sf_params("vina")
    box = {"center": rec["center"], "size": rec["size"]}

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- device-resident inputs (built before the timed region) ----
    types = np.unique(np.concatenate([l.types for l in ligs]))
    gs = make_gridset([rec], sfp, params.GRID_SPACING, params.OUT_OF_BOX_PENALTY, device=dev, lig_types=[types])
    lb = LigandBatch(ligs, dev)
    prob = Problem(gs, lb, torch.zeros(len(ligs), dtype=torch.long, device=dev), PairPotential(sfp, dev),
                   rec=pad_receptors([rec], dev))
    kp = B200KernelProblem(prob)
    bc = torch.tensor(rec["center"], dtype=torch.float32, device=dev)[None].expand(len(ligs), 3)
    bs = [rec["size"]] * len(ligs)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    if args.mc_variant:
        cfg = dict(cfg, autotune=False)
        kp.mc_variant = args.mc_variant

    def step(stats):
        kp.evals.zero_()
        dock_problem_kernel(prob, bc, bs, cfg, seed=0, stats=stats, kernel_factory=lambda p: kp)

    for _ in range(args.warmup):
        step({})
    barrier()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(vis.split(",")[local_rank] if vis else local_rank)
    launches0 = _lib.LAUNCHES[0]
    step_ms, mc_ms, evals, atom_evals = [], [], 0, 0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = {}
        e0.record()
        step(st)
        e1.record()
        torch.cuda.synchronize(dev)
        step_ms.append(e0.elapsed_time(e1))
        mc_ms.append(st["mc_ms"])
        evals += st["mc_evals"]            # the MC phase (the timed dominant launch) alone
        atom_evals += st["mc_atom_evals"]
    barrier()
    clk = clocks.stop()
    launches = _lib.LAUNCHES[0] - launches0
    t_rank = sum(step_ms)
    from adock_b200.distributed import max_over_ranks
    t_max = max_over_ranks(t_rank, device=dev) if world > 1 else t_rank
    value = args.ligands * world * args.steps / (t_max / 1e3)

    # ---- end to end through the public API from host arrays ----
    e2e = None
    if not args.no_e2e:
        st = {}
        dock_screen(rec, box, ligs, cfg, device=dev, stats=st)   # warm-up (allocator, module load)
        barrier()
        e2e_ms, h2d, d2h = [], 0, 0
        for _ in range(max(1, args.steps)):
            flush.zero_()
            st = {}
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = dock_screen(rec, box, ligs, cfg, device=dev, stats=st)
            e1.record()
            torch.cuda.synchronize(dev)
            e2e_ms.append(e0.elapsed_time(e1))
            h2d, d2h = st.get("h2d_bytes", 0), st.get("d2h_bytes", 0)
            assert len(res) == len(ligs) and all(len(r["affinity"]) >= 1 for r in res)
        t = sum(e2e_ms)
        if world > 1:
            t = max_over_ranks(t, device=dev)
        e2e = {"value": args.ligands * world * len(e2e_ms) / (t / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "spread": [args.ligands * world / (max(e2e_ms) / 1e3), args.ligands * world / (min(e2e_ms) / 1e3)],
               "repeats": len(e2e_ms)}

    # ---- roofline of the dominant kernel (MC + BFGS persistent kernel) ----
    peak, peak_kind = _peaks()
    mc_s = sum(mc_ms) / 1e3
    alg_bytes = atom_evals * 8 * 4           # 8 FP32 corner values gathered per atom evaluation
    achieved = alg_bytes / mc_s / 1e9
    tpa = _traffic_per_atom_eval()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "kernel": "mc_kernel",
            "traffic": (tpa * atom_evals / args.steps) if tpa is not None else None,
            "algorithmic_bytes_per_launch": alg_bytes / args.steps, "launch_ms": 1e3 * mc_s / args.steps}
    # the bound that applies to this gather/latency-bound kernel: warp-instruction issue (148 SMs x 4 schedulers x
    # 1 instruction per clock at the SM clock seen during the run), with the instructions per evaluation from ncu
    ipe = _profile_figure("warp_instructions_per_eval")
    if ipe is not None and clk.get("sm_mhz"):
        n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
        issue_peak = n_sm * 4 * clk["sm_mhz"] * 1e6
        issue = ipe * evals / mc_s
        roof["issue"] = {"achieved": issue / 1e9, "peak": issue_peak / 1e9, "unit": "G warp-instr/s",
                         "frac": issue / issue_peak, "instructions_per_eval": ipe}
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, shapes of the batched uneven workload)",
           "config": {"workload": WORKLOAD, "ligands_per_gpu": args.ligands, "chains": CHAINS, "mc_steps": args.mc_steps,
                      "l2": "flushed (256 MB write) between timed steps", "parallelism": f"ligand shards x{world}"},
           "value_spread": [args.ligands * world / (max(step_ms) / 1e3), args.ligands * world / (min(step_ms) / 1e3)],
           "evals_per_s": evals * world / mc_s, "mc_share_of_step": sum(mc_ms) / sum(step_ms),
           "roofline": roof, "clocks": clk, "gpu_launches": launches, "e2e": e2e,
           "mc_autotune": __import__("adock_b200.autotune", fromlist=["cached"]).cached()}
    if rank == 0 and world == 1 and not args.no_extras:
        out["grid_and_precision"] = _grid_and_precision(dev, ligs)
    variants = parse_variants(args.ab_variants)
    if rank == 0 and world == 1 and args.ab:
        from adock_b200 import synth
        from adock_b200.proposal import ab_compare
        train = synth.ligand_set(args.ab_train, (10, 60), (0, 15), seed0=100_000)
        held = synth.ligand_set(args.ab_eval, (10, 60), (0, 15), seed0=200_000)
        out["learned_proposal"] = ab_compare(rec, train, held, device=dev, learned=variants)
    if rank == 0 and world == 1 and args.screen:
        # screening shapes: the 8,000-atom receptor (30 A box, 81^3 maps), ligands with 8-80 heavy atoms and
        # 0-20 torsions; FP16 maps + learned proposal against the plain FP32 search at equal median gap
        from adock_b200 import synth
        from adock_b200.proposal import ab_compare
        rec2 = synth.config_receptor(2)
        train = synth.ligand_set(args.screen_train, (8, 80), (0, 20), seed0=300_000)
        held = synth.ligand_set(args.screen_eval, (8, 80), (0, 20), seed0=400_000)
        t0 = time.perf_counter()
        out["screening"] = ab_compare(rec2, train, held, device=dev, budgets=(250, 500, 1000, 2000, 4000),
                                      learned=parse_variants(args.screen_variants), log_cap=args.screen_log_cap)
        out["screening"]["wall_s"] = time.perf_counter() - t0
    if rank == 0 and world == 1 and not args.no_learned:
        out["learned_proposal"] = _learned_section(dev, args.learned_train, args.learned_eval)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = _cpu_baseline(ligs, rec, cfg)
    return out


def _learned_section(dev, n_train, n_eval):
    """The learned half of the metric on the screening shapes (the 8,000-atom receptor, 30 A box, 81^3 x 8 maps;
    ligands with 8-80 heavy atoms and 0-20 torsions), at reduced ligand counts: the proposal network is trained on
    the plain search's own moves from n_train fresh ligands (two self-training rounds, <= 2 M logged moves per
    collection; 4 candidate targets per learned step; 3-component translation mixture; 60 % of the steps learned
    before step 64, 30 % after), then FP16 maps + learned
    proposal and plain FP32 dock n_eval held-out ligands x 32 chains from the same Stage-A starts at several step
    budgets. Gap = a ligand's best energy minus the lowest energy any run
    found for it (an 8,000-step plain run included). Reported: ligands/s and energy evaluations/s of each method
    at the budget where its median gap reaches 0.1 kcal/mol (interpolated between budgets), and their ratio."""
    from adock_b200 import synth
    from adock_b200.proposal import ab_compare
    rec2 = synth.config_receptor(2)
    train = synth.ligand_set(n_train, (8, 80), (0, 20), seed0=300_000)
    held = synth.ligand_set(n_eval, (8, 80), (0, 20), seed0=400_000)
    t0 = time.perf_counter()
    ab = ab_compare(rec2, train, held, device=dev, budgets=(250, 500, 1000, 2000, 4000),
                    learned=[("learned_f16", 32, (0.6, 0.3, 64), "dagger2", 4, False, 3)], log_cap=2_000_000,
                    learned_budgets=(250, 500, 1000, 2000), plain_f16=False)
    wall = time.perf_counter() - t0
    interp = ab.get("interp_at_gap_0.1", {})

    def at_bar(m):
        r = interp.get(m)
        if not r:
            return None
        rows = sorted(ab["methods"][m], key=lambda x: x["steps"])
        near = min(rows, key=lambda x: abs(x["steps"] - r["steps"]))
        return {"steps": r["steps"], "ligands_per_s": r["ligands_per_s"], "evals_per_s": near["evals_per_s"]}

    plain, learned = at_bar("plain_f32"), at_bar("learned_f16")
    # the network's share of the learned search (features, GEMMs, sampling vs the MC launches), over its budgets
    lr = [r for r in ab["methods"]["learned_f16"] if "net_ms" in r]
    net_share = (sum(r["net_ms"] for r in lr) / sum(r["net_ms"] + r["mc_segments_ms"] for r in lr)) if lr else None
    return {"workload": (f"screening shapes: 8000-atom receptor, 30 A box, 81^3 x 8 maps; {n_eval} held-out ligands "
                         f"(8-80 heavy atoms, 0-20 torsions) x 32 chains; proposal trained on {n_train} fresh "
                         f"ligands (2 self-training rounds, 3-component translation mixture, 4 tries per learned step, "
                         f"learned fraction 0.6 before step 64 and 0.3 after)"),
            "gap_bar_kcal_mol": 0.1, "plain_f32": plain, "learned_f16": learned,
            "speedup_ligands_per_s_at_gap_0.1": (learned["ligands_per_s"] / plain["ligands_per_s"]
                                                 if plain and learned else None),
            "train_ms": {k: v["train_ms"] for k, v in ab["train"].items() if isinstance(v, dict)},
            "train_moves": ab["train"]["moves"], "wall_s": wall, "network_share_of_learned_search": net_share,
            "rows": {m: [{k: r[k] for k in ("steps", "median_gap", "mean_gap", "ligands_per_s", "evals_per_s")}
                         for r in rs] for m, rs in ab["methods"].items()}}


def _grid_and_precision(dev, ligs):
    """Map builder and map-precision figures on the 8,000-atom receptor (30 A box, 81^3): Vina maps for the 8
    ligand types and the fitted function's maps, timed with CUDA events; per-pose error of FP32/FP16/BF16 maps
    against float64 evaluation on 100k random poses of this batch's ligands."""
    import numpy as np
    import torch
    from scipy.spatial import cKDTree
    from adock_b200 import params, synth
    from adock_b200.grid import build_grid, build_grid_fit, grid_dims, prepare_grid, prepare_grid_fit
    from adock_b200.precision import precision_report
    rec2 = synth.config_receptor(2)
    sfp = params.sf_params("vina")
    o = rec2["center"] - rec2["size"] / 2
    n = grid_dims(rec2["size"], params.GRID_SPACING)
    lt = np.unique(np.concatenate([[0]] + [l.types for l in ligs]))
    spec = params.fitted_spec()
    pot = params.FittedPotential(spec, params.fitted_weights(), lt)
    rext = params.receptor_ext_types(rec2["rec_xyz"], rec2["rec_types"], spec)

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    ms_vina = timed(lambda: build_grid(rec2["rec_xyz"], rec2["rec_types"], sfp, o, params.GRID_SPACING, n, lt, device=dev))
    ms_fit = timed(lambda: build_grid_fit(rec2["rec_xyz"], rext, pot, o, params.GRID_SPACING, n, device=dev))
    # the kernels alone: launches back to back on prepared inputs (the calls above include the host preparation)
    lv, size_v, _ = prepare_grid(rec2["rec_xyz"], rec2["rec_types"], sfp, o, params.GRID_SPACING, n, lt, device=dev)
    lf, size_f, _ = prepare_grid_fit(rec2["rec_xyz"], rext, pot, o, params.GRID_SPACING, n, device=dev)
    out_v = torch.empty(size_v, device=dev)
    out_f = torch.empty(size_f, device=dev)
    kms_vina = timed(lambda: lv(out_v), reps=20)
    kms_fit = timed(lambda: lf(out_f), reps=20)
    # (point, receptor atom) pairs within the 8 A cutoff: the builder's algorithmic work per type
    axes = [o[d] + params.GRID_SPACING * np.arange(n[d]) for d in range(3)]
    pts = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    pairs = int(cKDTree(rec2["rec_xyz"]).count_neighbors(cKDTree(pts), 8.0 - 1e-6))
    pte = pairs * len(lt)
    return {"receptor": "8000 atoms, 60 A cube; 30 A box, %dx%dx%d points" % tuple(n), "types": len(lt),
            "vina_ms": ms_vina, "fitted_ms": ms_fit, "vina_kernel_ms": kms_vina, "fitted_kernel_ms": kms_fit,
            "point_atom_pairs": pairs,
            "vina_pair_type_evals_per_s": pte / (kms_vina / 1e3), "fitted_pair_type_evals_per_s": pte / (kms_fit / 1e3),
            "precision_100k_poses": precision_report(rec2, ligs, 100_000, device=dev)}


def _cpu_baseline(ligs, rec, cfg):
    """The reference's own search (stock driver and CPU kernels, baseline/_ref) on the host cores, on a 4-ligand
    quantile sample of the workload."""
    import torch
    A = _stock_reference()
    sample = _cpu_sample(ligs)
    if A is None:
        return {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                "sample": "unavailable: the reference package is not installed under baseline/_ref"}
    torch.set_num_threads(A.threads)
    prob = _reference_problem(A, rec, sample)
    _reference_search(A, prob, dict(cfg, mc_steps=20, mc_segment=20))     # compile + page in (untimed)
    dt, _ = _reference_search(A, prob, cfg)
    return {"value": len(sample) / dt, "unit": UNIT, "cores": A.threads, "kind": "reference",
            "sample": f"{len(sample)} ligands (heavy atoms {[p.n for p in sample]}) x {CHAINS} chains x "
                      f"{cfg['mc_steps']} steps, one full stock search, {dt:.1f} s"}


def parse_variants(spec):
    """Learned variants from "name:segment_steps:fraction[:training[:tries[:hint[:n_comp]]]],..." (fraction "0.3"
    or "0.6>0.3@64") as the tuples ``proposal.parse_learned`` reads."""
    from adock_b200.proposal import parse_frac
    out_v = []
    for v in spec.split(","):
        if not v:
            continue
        f = v.split(":")
        out_v.append((f[0], int(f[1]), parse_frac(f[2])) + ((f[3],) if len(f) > 3 else ())
                     + ((int(f[4]),) if len(f) > 4 else ()) + ((f[5] in ("1", "hint"),) if len(f) > 5 else ())
                     + ((int(f[6]),) if len(f) > 6 else ()))
    return out_v


def run_screen_full(args):
    """The full-form screening workload (configs of the screening run: FP16 maps, learned proposal, 32 chains per
    ligand, ligands with 8-80 heavy atoms and 0-20 torsions against the 8,000-atom receptor) as one batch, against
    the plain FP32 search of the same batch; the reference's CPU search on a quantile sample of the first 256
    ligands at the plain budget."""
    import numpy as np
    import torch
    from adock_b200 import params, synth
    from adock_b200.proposal import full_screen
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rec2 = synth.config_receptor(2)
    nw = min(16, os.cpu_count() or 1)     # the generator is Python; the seeds are split over processes
    train = synth.ligand_set(args.screen_train, (8, 80), (0, 20), seed0=300_000, workers=nw)
    ligs = synth.ligand_set(args.screen_full_ligands, (8, 80), (0, 20), seed0=700_000, workers=nw)
    variant = parse_variants(args.screen_variants)[0]
    clocks = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    t0 = time.perf_counter()
    steps_l = tuple(int(x) for x in args.screen_full_learned_steps.split(",") if x)
    res = full_screen(rec2, train, ligs, variant, device=dev, learned_steps=steps_l,
                      plain_steps=args.screen_full_plain_steps, n_sub=args.screen_full_subset,
                      log_cap=args.screen_log_cap)
    res["wall_s"] = time.perf_counter() - t0
    res["clocks"] = clocks.stop()
    out = {"metric": "ligands docked/s at equal median best-energy gap: learned FP16 vs plain FP32 search", "unit": UNIT,
           "workload": f"full-form screening: {len(ligs)} ligands (8-80 heavy atoms, 0-20 torsions) x 32 chains vs "
                       "the 8,000-atom receptor (30 A box, 81^3 x 8 maps); learned FP16 vs plain FP32",
           "data": "synthetic (seeded)", "screen_full": res}
    if args.screen_full_cpu > 0:
        A = _stock_reference()
        if A is None:
            out["cpu_baseline"] = {"value": None, "sample": "unavailable: the reference package is not installed"}
        else:
            torch.set_num_threads(A.threads)
            sub = ligs[:256]
            order = sorted(range(len(sub)), key=lambda i: (sub[i].n, i))
            n = args.screen_full_cpu
            sample = [sub[order[int(len(order) * (j + 0.5) / n)]] for j in range(n)]
            cfg = params.workload_preset(32, args.screen_full_plain_steps)
            prob = _reference_problem(A, rec2, sample)
            _reference_search(A, prob, dict(cfg, mc_steps=20, mc_segment=20))    # compile + page in (untimed)
            dt, _ = _reference_search(A, prob, cfg)
            out["cpu_baseline"] = {"value": len(sample) / dt, "unit": UNIT, "cores": A.threads, "kind": "reference",
                                   "sample": f"{len(sample)} ligands at the quantiles of the heavy-atom count of the "
                                             f"first 256 x 32 chains x {cfg['mc_steps']} steps (the plain budget), "
                                             f"one full stock search, {dt:.1f} s"}
    return out


def main():
    args = _args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # the longest gap between two collectives is the warm-up (autotune + 3 steps, well under a minute)
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=180))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.screen_full:
        out = run_screen_full(args) if rank == 0 else None
    else:
        out = run_ours(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
