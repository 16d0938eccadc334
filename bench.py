#!/usr/bin/env python
"""Benchmark: right-hand sides solved per second to 1e-8 relative residual.

Workload (default): the batched + mixed-precision MT configuration with
topography -- ~1.5M tets, 8 frequencies log-spaced in [1e-3, 100] Hz x 2
polarisations = 16 right-hand sides solved as one block (synthetic seeded
mesh/model from emfem_b200.meshgen).  One step = the hot path over that
batch: assemble_matrix, AMS setup, MT right-hand sides, block
FGMRES(FCG(AMS)) solve with FP64 outer iterations and an FP32 AMS.

value  : RHS/s with inputs resident on the device (device-timed, CUDA events)
e2e    : RHS/s through the host-buffer C ABI (emg_assemble_rhs_mt_block +
         emg_solve_block), host<->device copies inside the timed region
plain_fp64 : the per-RHS FP64 drop-in (real-form FGMRES, per-frequency AMS
         setup, zero guess) on every column of the same workload, for the ratio
field_err_vs_fp64 : the headline solution against an FP64 block solve of the
         same columns to 1e-11: receiver E/H, MT rho_a/phase, whole solution
dual   : the dual solves (one per frequency, rtol 1e-6), timed separately
roofline : the edge-level FP32 SpMM inside the AMS (the launch shape with
         the largest share of device time), achieved algorithmic GB/s from
         CUDA events around its launches in one profiled step after the timed
         region; traffic from the committed ncu capture's traffic ratio
cpu_baseline : the CPU oracle (restatement of the reference path) on a bounded
         sample of the full-size workload (assembly, AMS setup, one FGMRES
         iteration), extrapolated by the inner iteration count of complete
         oracle solves of it; rank 0, N=1 only
Under torchrun (N > 1) every rank runs the timed replica steps, the profiled
step and e2e; plain_fp64, field_err_vs_fp64, dual and warm_start are N=1
reports and are left out there.

--impl reference times complete CPU-oracle solves (the reference's own
MPI/PETSc binary cannot be built in this image), one column per step, on the
workload's model at mesh scale --ref-scale, and prints the same line with
"impl": "reference"; its cpu_baseline.extrapolated holds the full-size
estimate (the bounded sample above).
"""

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RHS solved/s at 1e-8 residual: mixed+batched+warm-start vs plain FP64 (1 B200)"
UNIT = "RHS/s"


def log(msg):
    print("[bench %.0fs] %s" % (time.perf_counter() - _T0, msg), file=sys.stderr, flush=True)


_T0 = time.perf_counter()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--plain-freqs", type=int, default=-1,
                    help="frequencies timed on the plain FP64 path (-1: all of them)")
    ap.add_argument("--plain-tx", type=int, default=2, help="CSEM: transmitters per frequency on the plain path")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP64 reference solve")
    ap.add_argument("--no-dual", action="store_true", help="skip the timed dual solves")
    ap.add_argument("--ref-scale", type=float, default=0.03,
                    help="--impl reference: mesh scale at which complete oracle solves are timed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-warm", action="store_true", help="skip the learned warm-start arm")
    ap.add_argument("--warm-steps", type=int, default=300, help="Adam steps of the warm-start network")
    ap.add_argument("--warm-batch", type=int, default=65536, help="samples per Adam step")
    ap.add_argument("--breakdown", action="store_true", help="print per-phase host timings to stderr")
    ap.add_argument("--no-profile", action="store_true",
                    help="skip the profiled step and the phase step after the timed region (no roofline)")
    ap.add_argument("--no-phases", action="store_true", help="skip the phase step after the timed region")
    ap.add_argument("--options", default="", help="extra solver options (process_options text)")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


class Cols:
    """The workload's right-hand sides: MT columns (frequency x polarisation)
    or CSEM columns (frequency x transmitter), with the source id of each
    column (polarisation or transmitter) and, for CSEM, its position."""

    def __init__(self, prob, idx=None):
        self.freqs = np.asarray(prob.survey.freqs, dtype=np.float64)
        self.kind = prob.survey.kind
        nf = self.freqs.size
        if self.kind == "mt":
            self.colf = np.repeat(self.freqs, 2)
            self.src = np.tile(np.array([0, 1], dtype=np.int32), nf)
            self.modes = np.where(self.src == 0, -1, -2).astype(np.int32)
            self.tx = None
        else:
            ntx = len(prob.survey.tx)
            self.colf = np.repeat(self.freqs, ntx)
            self.src = np.tile(np.arange(ntx, dtype=np.int32), nf)
            self.modes = None
            self.tx = np.asarray(prob.survey.tx, dtype=np.float64)[self.src]
        if idx is not None:
            self.colf, self.src = self.colf[idx], self.src[idx]
            self.modes = None if self.modes is None else self.modes[idx]
            self.tx = None if self.tx is None else self.tx[idx]

    @property
    def k(self):
        return self.colf.size

    @property
    def pos(self):
        return None if self.tx is None else self.tx[:, :3]

    def fidx(self):
        return np.searchsorted(self.freqs, self.colf)

    def assemble_dev(self, ctx, ptr):
        if self.kind == "mt":
            ctx.assemble_rhs_mt_block_dev(self.colf, self.modes, ptr)
        else:
            ctx.assemble_rhs_csem_block_dev(self.colf, self.tx, ptr)

    def assemble_host(self, ctx, scratch):
        """the right-hand sides as a host array (device kernels, then D2H)"""
        if self.kind == "mt":
            return ctx.assemble_rhs_mt_block(self.colf, self.modes)
        self.assemble_dev(ctx, scratch.data_ptr())
        return scratch.cpu().numpy()


def roofline_traffic(bin_name, algo_bytes_per_launch):
    """DRAM traffic per launch of the profiled kernel from the committed ncu
    summary (profiles/<bin>_traffic.txt).  The capture is one launch of a
    smaller case of the same kernel; its traffic / algorithmic-bytes ratio,
    applied to this run's average algorithmic bytes per launch, gives the
    traffic of a launch here (traffic grows with rows and nonzeros)."""
    path = os.path.join(ROOT, "profiles", bin_name + "_traffic.txt")
    vals = {}
    try:
        with open(path) as f:
            for line in f:
                if ":" in line and not line.startswith("#"):
                    k, v = line.split(":", 1)
                    vals[k.strip()] = float(v)
    except OSError:
        return None, None
    if "traffic_over_algorithmic" in vals:
        return vals["traffic_over_algorithmic"] * algo_bytes_per_launch, vals["traffic_over_algorithmic"]
    return vals.get("traffic_bytes_per_launch"), None


# ----------------------------------------------------------------------------
# learned warm start on the workload's columns
# ----------------------------------------------------------------------------
def warm_start_arm(args, ctx, cols, rhs, ne, infos_single):
    """Two-stage schedule: the columns of every other frequency (anchors) are
    solved from zero; the warm-start network is trained on them; the remaining
    columns start from its guess.  Timed as a whole step (assembly and
    right-hand sides included); the target columns are also solved from zero
    and from the log-f interpolation alone (A/B)."""
    import torch
    fi = cols.fidx()
    ia = np.nonzero(fi % 2 == 0)[0]
    it = np.nonzero(fi % 2 == 1)[0]
    ka, kt = ia.size, it.size
    pos_a = None if cols.pos is None else cols.pos[ia]
    pos_t = None if cols.pos is None else cols.pos[it]
    sa = torch.zeros((ne, ka), dtype=torch.complex128, device="cuda")
    xa = torch.zeros_like(sa)
    st = torch.zeros((ne, kt), dtype=torch.complex128, device="cuda")
    xt = torch.zeros_like(st)
    ia_d = torch.from_numpy(ia).to("cuda")
    it_d = torch.from_numpy(it).to("cuda")
    fa, fsa, ft, fst = cols.colf[ia], cols.src[ia], cols.colf[it], cols.src[it]
    rec = {}

    def two_stage():
        ctx.warm_start_reset()
        t0 = time.perf_counter()
        ctx.assemble_matrix(0)
        cols.assemble_dev(ctx, rhs.data_ptr())
        torch.index_select(rhs, 1, ia_d, out=sa)
        torch.index_select(rhs, 1, it_d, out=st)
        torch.cuda.synchronize()
        inf_a = ctx.solve_block_dev(fa, sa.data_ptr(), xa.data_ptr(), rtol=1e-8, max_it=200, inner_fp32=True)
        t1 = time.perf_counter()
        loss = ctx.warm_start_train(fa, fsa, xa.data_ptr(), src_pos=pos_a, steps=args.warm_steps,
                                    batch=args.warm_batch, lr=2e-3, seed=11)
        ctx.warm_start_predict(fa, fsa, xa.data_ptr(), ft, fst, xt.data_ptr(), src_pos=pos_a, tsrc_pos=pos_t,
                               network=2)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        inf_t = ctx.solve_block_dev(ft, st.data_ptr(), xt.data_ptr(), rtol=1e-8, max_it=200, inner_fp32=True,
                                    use_guess=True)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        rec.update(loss=loss, losses=ctx.warm_start_losses(), inf_a=inf_a, inf_t=inf_t,
                   r0=ctx.last_initial_residuals(kt), t_anchor=t1 - t0,
                   t_net=t2 - t1, t_target=t3 - t2)
        return t3 - t0

    log("warm-start arm: %d anchor columns, %d predicted" % (ka, kt))
    for _ in range(max(1, min(args.warmup, 2))):
        two_stage()
    n_t = max(1, min(args.steps, 3))
    times = [two_stage() for _ in range(n_t)]
    t_step = float(np.mean(times))
    # A/B on the target columns: zero start and the interpolation alone
    ab = {}
    for arm in ("zero", "interp", "network", "quadratic"):
        xt.zero_()
        if arm != "zero":
            ctx.warm_start_predict(fa, fsa, xa.data_ptr(), ft, fst, xt.data_ptr(), src_pos=pos_a, tsrc_pos=pos_t,
                                   network={"interp": 0, "network": 1, "quadratic": 3}[arm])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        inf = ctx.solve_block_dev(ft, st.data_ptr(), xt.data_ptr(), rtol=1e-8, max_it=200, inner_fp32=True,
                                  use_guess=(arm != "zero"))
        torch.cuda.synchronize()
        ab[arm] = dict(outer_its=[i.outer_its for i in inf], inner_its=int(sum(i.inner_its for i in inf[:1])),
                       initial_res=[float(v) for v in ctx.last_initial_residuals(kt)],
                       block_ms=1e3 * (time.perf_counter() - t0))
    single_ms = 1e3 * (infos_single[0].seconds if infos_single else float("nan"))
    out = {
        "network": ("per-edge MLP, 13 inputs (2 neighbour-frequency values scaled per edge, log resistivities, "
                    "log length, direction cosines, log distance to the source, log f, tau), 3 hidden layers of 64 "
                    "with GELU, output the curvature in log f (q = (lg f - lg f_a)(lg f - lg f_b) times it corrects the log-f "
                    "interpolation); BF16 weights, FP32 accumulation, tcgen05 "
                    "forward and backward kernels, Adam"),
        "schedule": ("anchor columns (frequencies %s, every source) solved from zero; network trained on them "
                     "(%d Adam steps of %d samples); the other %d columns solved from its guess (the network's "
                     "correction where its training loss is a quarter of the interpolation's, else the quadratic "
                     "log-f interpolation)"
                     % ([float(f) for f in cols.freqs[::2]], args.warm_steps, args.warm_batch, kt)),
        "value": cols.k / t_step, "unit": UNIT, "ms_per_step": 1e3 * t_step, "steps_timed": n_t,
        "timing": "host wall clock around the whole two-stage step (assembly, right-hand sides, both solves, "
                  "training and prediction), after %d untimed steps" % max(1, min(args.warmup, 2)),
        "anchor_block_ms": 1e3 * rec["t_anchor"], "network_ms": 1e3 * rec["t_net"],
        "target_block_ms": 1e3 * rec["t_target"], "train_loss": rec["loss"],
        "train_loss_interpolation": rec["losses"][1],
        "guess": ("network" if 0 <= rec["losses"][0] <= 0.25 * rec["losses"][1] else
                  "quadratic log-f interpolation where three anchors bracket the target, linear elsewhere (the "
                  "network's training loss was above a quarter of the linear interpolation's)"),
        "anchor_outer_its": [i.outer_its for i in rec["inf_a"]],
        "anchor_inner_its": int(rec["inf_a"][0].inner_its),
        "target_outer_its_network": [i.outer_its for i in rec["inf_t"]],
        "target_inner_its_network": int(rec["inf_t"][0].inner_its),
        "target_initial_res_network": [float(v) for v in rec["r0"]],
        "target_true_rel_res_max": max(i.true_rel_res for i in rec["inf_t"]),
        "converged": all(i.reason == 0 for i in list(rec["inf_a"]) + list(rec["inf_t"])),
        "target_outer_its_zero": ab["zero"]["outer_its"], "target_inner_its_zero": ab["zero"]["inner_its"],
        "target_block_ms_zero": ab["zero"]["block_ms"],
        "target_outer_its_interp": ab["interp"]["outer_its"], "target_inner_its_interp": ab["interp"]["inner_its"],
        "target_initial_res_interp": ab["interp"]["initial_res"], "target_block_ms_interp": ab["interp"]["block_ms"],
        "target_outer_its_network_forced": ab["network"]["outer_its"],
        "target_inner_its_network_forced": ab["network"]["inner_its"],
        "target_initial_res_network_forced": ab["network"]["initial_res"],
        "target_block_ms_network_forced": ab["network"]["block_ms"],
        "target_outer_its_quadratic": ab["quadratic"]["outer_its"],
        "target_initial_res_quadratic": ab["quadratic"]["initial_res"],
        "target_block_ms_quadratic": ab["quadratic"]["block_ms"],
        "single_block_solve_ms": single_ms,
    }
    log("warm start: %.1f ms/step; target its guess %s zero %s interp %s network %s quadratic %s" % (
        out["ms_per_step"], out["target_outer_its_network"], out["target_outer_its_zero"],
        out["target_outer_its_interp"], out["target_outer_its_network_forced"], out["target_outer_its_quadratic"]))
    return out


# ----------------------------------------------------------------------------
# accuracy of a block solution against a reference block at the receivers
# ----------------------------------------------------------------------------
def field_accuracy(ctx, E, cols, x, xref, rx, rx_tets, plain_fields=None):
    """Receiver E/H (interpolate_fields on the device), for MT the apparent
    resistivity and phase (calculate_response_mt's AP pair), and the whole
    solution of each column against the converged FP64 block; with
    plain_fields ({column: (E, H)} of the per-RHS FP64 path at the same
    rtol, the reference's own method) the same errors of that path."""
    colf = cols.colf
    Eh, Hh = ctx.interpolate_fields_block_dev(colf, x.data_ptr(), rx, rx_tets)
    Er, Hr = ctx.interpolate_fields_block_dev(colf, xref.data_ptr(), rx, rx_tets)

    def rel_rows(a, b):
        return np.abs(a - b).max(axis=-1) / np.maximum(np.abs(b).max(axis=-1), 1e-300)

    eE, eH = rel_rows(Eh, Er), rel_rows(Hh, Hr)          # (nrx, k)
    import torch
    dof = (torch.abs(x - xref).amax(dim=0) / torch.abs(xref).amax(dim=0)).cpu().numpy()
    nrx = rx.shape[0]

    def mt_errors(Ea, Ha):
        otype = np.array([E.api.R_XY_AP, E.api.R_YX_AP] * nrx, dtype=np.int32)
        ridx = np.repeat(np.arange(nrx, dtype=np.int32), 2)
        drho, dph = 0.0, 0.0
        for f in cols.freqs:
            jx = [j for j in range(colf.size) if colf[j] == f]
            if len(jx) != 2 or Ea[jx[0]] is None or Ea[jx[1]] is None:
                continue
            a = E.calculate_response_mt(f, np.stack([Ea[jx[0]], Ha[jx[0]], Ea[jx[1]], Ha[jx[1]]], 1), otype, ridx)
            b = E.calculate_response_mt(f, np.stack([Er[:, jx[0]], Hr[:, jx[0]], Er[:, jx[1]], Hr[:, jx[1]]], 1),
                                        otype, ridx)
            drho = max(drho, float(np.abs(np.expm1(a.real - b.real)).max()))
            dph = max(dph, float(np.abs(np.degrees(np.angle(np.exp(1j * (a.imag - b.imag))))).max()))
        return drho, dph

    drho, dph = (None, None)
    if cols.kind == "mt":
        drho, dph = mt_errors([Eh[:, j] for j in range(colf.size)], [Hh[:, j] for j in range(colf.size)])
    out = {"receivers": int(nrx), "E_max_rel": float(eE.max()), "H_max_rel": float(eH.max()),
           "E_max_rel_per_column": [float(v) for v in eE.max(axis=0)],
           "H_max_rel_per_column": [float(v) for v in eH.max(axis=0)],
           "solution_max_rel_per_column": [float(v) for v in dof],
           "rho_a_max_rel": drho, "phase_max_deg": dph,
           "meets_1e-6_receiver_bar": bool(eE.max() <= 1e-6 and eH.max() <= 1e-6)}
    ok = True
    if plain_fields:
        pE = [None] * colf.size
        pH = [None] * colf.size
        for j, (e_, h_) in plain_fields.items():
            pE[j], pH[j] = e_, h_
        cols_p = sorted(plain_fields)
        peE = {j: float(rel_rows(pE[j], Er[:, j]).max()) for j in cols_p}
        peH = {j: float(rel_rows(pH[j], Hr[:, j]).max()) for j in cols_p}
        out["per_rhs_fp64_at_rtol_1e-8"] = {
            "columns": cols_p, "E_max_rel_per_column": [peE[j] for j in cols_p],
            "H_max_rel_per_column": [peH[j] for j in cols_p]}
        if cols.kind == "mt":
            out["per_rhs_fp64_at_rtol_1e-8"]["rho_a_max_rel"], out["per_rhs_fp64_at_rtol_1e-8"]["phase_max_deg"] = \
                mt_errors(pE, pH)
        # the same accuracy class: the worst receiver error over the columns
        # no more than twice the per-RHS FP64 method's worst at the same rtol
        wE, wH = max(peE.values()), max(peH.values())
        ok = eE[:, cols_p].max() <= max(2 * wE, 1e-6) and eH[:, cols_p].max() <= max(2 * wH, 1e-6)
        out["per_rhs_fp64_at_rtol_1e-8"]["E_max_rel"], out["per_rhs_fp64_at_rtol_1e-8"]["H_max_rel"] = wE, wH
        out["columns_within_2x_of_per_rhs"] = {
            "E": int(sum(eE[:, j].max() <= max(2 * peE[j], 1e-6) for j in cols_p)),
            "H": int(sum(eH[:, j].max() <= max(2 * peH[j], 1e-6) for j in cols_p)), "of": len(cols_p)}
    if drho is not None:
        ok = ok and drho <= 1e-3 and dph <= 0.05
    out["bar"] = ("receiver E and H (per receiver, max component error over the largest component) against the "
                  "converged FP64 fields: the worst over the columns no more than twice the per-RHS FP64 path's "
                  "worst at the same rtol (floor 1e-6); MT rho_a 0.1 %, phase 0.05 deg")
    out["meets_bar"] = bool(ok)
    return out


# ----------------------------------------------------------------------------
# CPU oracle baseline (bounded sample)
# ----------------------------------------------------------------------------
def cpu_sample(prob, n_rhs_per_setup=2, max_outer=1):
    """Times the oracle on one frequency of the workload: assembly, AMS setup
    and `max_outer` FGMRES iterations of one RHS.  Returns the measured times."""
    import oracle as O
    threads = O.num_threads(0)
    m = O.Mesh(prob.mesh)
    rp, ci = O.sparsity(m)
    f = float(prob.survey.freqs[0])
    t0 = time.perf_counter()
    Cv, Mv, bdr = O.assemble(m, prob.model, f, rp, ci)
    t_asm = time.perf_counter() - t0
    obg = O.background_model(m, prob.model)
    t0 = time.perf_counter()
    sr, si = O.rhs_mt(m, prob.model, f, -1, obg, bdr)
    t_rhs = time.perf_counter() - t0
    er, ei, its, st = O.solve(m, rp, ci, Cv, Mv, sr, si, 1e-8, max_outer)
    return dict(threads=threads, t_asm=t_asm, t_rhs=t_rhs, t_setup=float(st[2]), t_fgmres=float(st[3]),
                outer=int(its), inner=int(st[1]))


def cpu_calibration(cfg):
    """Iteration counts of full oracle solves on this workload (committed)."""
    path = os.path.join(ROOT, "oracle", "calibration_cfg%d.json" % cfg)
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def cpu_rhs_per_s(sample, inner_per_rhs):
    t_inner = sample["t_fgmres"] / max(sample["inner"], 1)
    per_rhs = (sample["t_asm"] + sample["t_setup"]) / 2.0 + sample["t_rhs"] + inner_per_rhs * t_inner
    return 1.0 / per_rhs, per_rhs


def oracle_column_solve(O, m, rp, ci, prob, obg, cols, j):
    """One complete oracle solve of column j: assembly, AMS setup, RHS and
    FGMRES(FCG(AMS)) to 1e-8 (the reference's per-task sequence)."""
    f = float(cols.colf[j])
    t0 = time.perf_counter()
    Cv, Mv, bdr = O.assemble(m, prob.model, f, rp, ci)
    if cols.kind == "mt":
        sr, si = O.rhs_mt(m, prob.model, f, int(cols.modes[j]), obg, bdr)
    else:
        sr, si = O.rhs_csem(m, f, cols.tx[j])
    er, ei, its, st = O.solve(m, rp, ci, Cv, Mv, sr, si, 1e-8, 200)
    return time.perf_counter() - t0, int(its), int(st[1]), float(st[0])


def reference_arm(args):
    world, rank, local = dist_setup()
    if rank != 0:
        barrier(world)
        return
    import oracle as O
    from emfem_b200 import meshgen as mg
    # complete oracle solves, one column per step, on the workload at a mesh
    # scale where one solve takes seconds (a full-size column takes ~15 min)
    prob = mg.config(args.config, args.ref_scale)
    cols = Cols(prob)
    m = O.Mesh(prob.mesh)
    rp, ci = O.sparsity(m)
    obg = O.background_model(m, prob.model) if cols.kind == "mt" else None
    threads = O.num_threads(0)
    for i in range(args.warmup):
        oracle_column_solve(O, m, rp, ci, prob, obg, cols, i % cols.k)
    times, its = [], []
    for i in range(args.steps):
        t, outer, inner, res = oracle_column_solve(O, m, rp, ci, prob, obg, cols, i % cols.k)
        times.append(t)
        its.append((outer, inner, res))
    v = len(times) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": prob.name, "scale": args.ref_scale, "tets": prob.mesh.n_tets,
                   "edges": prob.mesh.n_edges, "rhs_per_step": 1, "rtol": 1e-8},
        "outer_its": [o for o, _, _ in its], "inner_its": [i for _, i, _ in its],
        "true_rel_res_max": max(r for _, _, r in its),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": ("CPU oracle (C++ restatement of the reference path: assembly, AMS setup, MT RHS, "
                                    "real-form FGMRES(FCG(AMS)) to 1e-8; the PETSc/hypre binary cannot be built "
                                    "here), one complete solve of one column per step, columns in turn, on the "
                                    "workload's model at mesh scale %g (%d tets; the full-size mesh has about %d)"
                                    % (args.ref_scale, prob.mesh.n_tets, int(prob.mesh.n_tets / args.ref_scale)))},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    # the full-size workload, estimated (not timed end to end): assembly, AMS
    # setup and one FGMRES iteration of the oracle at --scale, scaled by the
    # inner iteration count of complete oracle solves of it
    if not args.no_cpu_baseline:
        try:
            full = mg.config(args.config, args.scale)
            sm = cpu_sample(full)
            cal = cpu_calibration(args.config)
            inner = cal["inner_per_rhs"] if cal else 30 * sm["inner"]
            ve, _ = cpu_rhs_per_s(sm, inner)
            line["cpu_baseline"]["extrapolated"] = {
                "value": ve, "unit": UNIT, "workload": full.name, "tets": full.mesh.n_tets,
                "edges": full.mesh.n_edges, "cores": sm["threads"],
                "sample": ("assembly %.2fs, AMS setup %.2fs, MT RHS %.2fs, %d FGMRES iteration(s) with %d inner FCG "
                           "iterations in %.2fs at full size; RHS/s = 1/((asm+setup)/2 + rhs + %.1f inner its per "
                           "RHS (%s) x time per inner iteration): an estimate, not an end-to-end time"
                           % (sm["t_asm"], sm["t_setup"], sm["t_rhs"], sm["outer"], sm["inner"], sm["t_fgmres"],
                              inner, "committed complete oracle solves of this workload" if cal else
                              "30 x the sampled count"))}
        except Exception as ex:  # the estimate must not kill the line
            line["cpu_baseline"]["extrapolated"] = {"value": None, "sample": "failed: %s" % ex}
    print(json.dumps(line), flush=True)
    barrier(world)


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def ours(args):
    world, rank, local = dist_setup()
    import torch
    import emfem_b200 as E
    from emfem_b200 import meshgen as mg

    torch.cuda.set_device(local)
    prob = mg.config(args.config, args.scale)
    cols = Cols(prob)
    freqs, colf = cols.freqs, cols.colf
    K = colf.size
    ctx = E.EMContext(local)
    if args.options:
        ctx.process_options(args.options)
    ctx.set_mesh(prob.mesh)
    ctx.set_model(prob.model)
    ctx.set_frequencies(freqs)
    ctx.create_linear_system(-3 if cols.kind == "mt" else 0)
    if cols.kind == "mt":
        ctx.set_background(*mg.background_model(prob.mesh, prob.model))
    ne = prob.mesh.n_edges
    rhs = torch.zeros((ne, K), dtype=torch.complex128, device="cuda")
    x = torch.zeros((ne, K), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    infos_last = []
    breakdown = {}

    def step():
        nonlocal infos_last
        t0 = time.perf_counter()
        ctx.assemble_matrix(0)
        t1 = time.perf_counter()
        cols.assemble_dev(ctx, rhs.data_ptr())
        t2 = time.perf_counter()
        infos_last = ctx.solve_block_dev(colf, rhs.data_ptr(), x.data_ptr(), rtol=1e-8, max_it=200,
                                         inner_fp32=True)
        t3 = time.perf_counter()
        su = ctx.last_kernel_ms("block_setup") / 1e3
        for k, v in (("assemble", t1 - t0), ("rhs", t2 - t1), ("ams_setup", su), ("solve", t3 - t2 - su)):
            breakdown[k] = breakdown.get(k, 0.0) + v
        for k in ("setup_edge", "setup_gtb", "setup_nodal", "setup_amg", "setup_upload", "setup_columns"):
            try:
                breakdown[k] = breakdown.get(k, 0.0) + ctx.last_kernel_ms(k) / 1e3
            except Exception:
                pass

    log("problem %s: %d tets, %d edges; warm-up %d steps" % (prob.name, prob.mesh.n_tets, ne, args.warmup))
    for i in range(args.warmup):
        step()
        log("warm-up step %d: %s outer its %s" % (i, {k: round(v, 2) for k, v in breakdown.items()},
                                                  [inf.outer_its for inf in infos_last]))
    breakdown.clear()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    log("timed region: %d steps" % args.steps)
    clocks = Clocks(local)
    clocks.start()
    l0 = E.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    launches = E.launch_count() - l0
    clk = clocks.stop()
    timed_breakdown = {k: round(v / args.steps, 3) for k, v in breakdown.items()}
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, world)
    barrier(world)
    ms_step = ms / args.steps
    value = world * K * args.steps / (ms / 1e3)
    log("timed: %.1f ms/step" % ms_step)
    # kernel attribution: one more step with the event profiler on (it runs
    # the AMS launch by launch, so it stays out of the timed region)
    bins, phases, prof_step_s = {}, None, 0.0
    if not args.no_profile:
        E.profile_enable(True)
        tp0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        prof_step_s = time.perf_counter() - tp0
        for b in ("spmm_edge_fp32", "spmm_edge_fp64", "spmm_nodal_fp32", "spmm_nodal_fp64", "vcycle_fused_fp32"):
            n, t, by = E.profile_get(b)
            bins[b] = (n, t, by)
        E.profile_enable(False)
        log("profiled step: %.1f s" % prof_step_s)
    if not args.no_profile and not args.no_phases:
        # solver phases with graphs and fused launches kept: events around the
        # outer FGMRES, each inner FCG solve, each AMS application and each FP64
        # operator apply
        E.profile_enable(2)
        step()
        torch.cuda.synchronize()
        phases = {}
        for b in ("phase_fgmres", "phase_fcg", "phase_ams", "phase_opB"):
            n, t, _ = E.profile_get(b)
            phases[b[6:]] = {"count": n, "ms": round(t, 2)}
        E.profile_enable(False)
        log("phases: %s" % phases)
    infos_headline = list(infos_last)

    # ---- learned warm start: anchors, training, predicted remainder ---------
    warm = None
    # the side arms (warm start, dual, plain FP64, accuracy) are N=1 reports;
    # under torchrun every rank would repeat them, so N>1 runs skip them
    single = world == 1
    if single and not args.no_warm and freqs.size >= 3:
        warm = warm_start_arm(args, ctx, cols, rhs, ne, infos_headline)

    rx = np.asarray(prob.survey.rx, dtype=np.float64)
    rx_tets = ctx.find_cell_around_point(rx)
    # ---- dual solves (rtol 1e-6), timed separately ----------------------------
    dual = None
    if single and not args.no_dual and (rx_tets >= 0).all():
        log("dual solves")
        kd = freqs.size
        d = torch.zeros((ne, kd), dtype=torch.complex128, device="cuda")
        xd = torch.zeros_like(d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.assemble_rhs_dual_block_dev(kd, rx, d.data_ptr())
        inf_d = ctx.solve_block_dev(freqs, d.data_ptr(), xd.data_ptr(), rtol=1e-6, max_it=100, inner_fp32=True)
        torch.cuda.synchronize()
        td = time.perf_counter() - t0
        floors = ctx.last_residual_floors(kd)
        dual = {"value": kd / td, "unit": "RHS/s", "rhs": kd, "rtol": 1e-6, "max_it": 100, "seconds": td,
                "outer_its": [i.outer_its for i in inf_d], "true_rel_res": [i.true_rel_res for i in inf_d],
                "fp64_residual_floor": [float(f) for f in floors],
                "stopped_at_floor": [bool(i.reason == E.api.EMG_STOPPED_AT_FLOOR) for i in inf_d],
                "converged": all(i.reason in (0, E.api.EMG_STOPPED_AT_FLOOR) for i in inf_d),
                "floor_note": ("a point-source dual right-hand side at low frequency drives a static gradient field "
                               "in the air whose FP64 residual cannot fall below u || |b| + |A||x| || / ||b|| "
                               "(u = 2^-53); such a column stops there (EMG_STOPPED_AT_FLOOR) instead of running "
                               "to max_it as the reference's KSP would"),
                "timing": ("host wall clock around the device dual right-hand sides (one per frequency, "
                           "src/em_fwd.cc:1354-1356) and their block solve, which reuses the primal block's "
                           "AMS setup")}
        del d, xd
    conv = [(i.true_rel_res, i.outer_its) for i in infos_headline]
    all_conv = all(i.reason == 0 and i.true_rel_res <= 1e-8 for i in infos_headline)
    # the roofline kernel is the edge-level FP32 SpMM of the AMS: the launch shape with
    # the largest share of device time in the committed launch list (profiles/), and the
    # one kernel that streams HBM; the nodal-level SpMMs (many small, L2-resident launch
    # shapes, bound by dependent steps) are reported beside it as a share
    dom = "spmm_edge_fp32"
    n_l, t_l, b_l = bins.get(dom, (0, 0.0, 0.0))
    peak, peak_kind = peaks()
    achieved = (b_l / max(n_l, 1)) / ((t_l / max(n_l, 1)) * 1e-3) / 1e9 if n_l else 0.0
    traffic, traffic_ratio = roofline_traffic(dom, b_l / max(n_l, 1))
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "algorithmic_bytes_per_launch": b_l / max(n_l, 1), "launches": n_l,
            "avg_launch_us": 1e3 * t_l / max(n_l, 1),
            "traffic_source": ("ncu dram bytes / algorithmic bytes = %.3f on the committed capture "
                               "(profiles/%s_traffic.txt), times this run's algorithmic bytes per launch"
                               % (traffic_ratio, dom)) if traffic_ratio else None,
            "measured": "CUDA events around every launch of the kernel during one profiled step of this "
                        "workload (launch by launch) right after the timed region",
            "share_of_profiled_step": t_l / (prof_step_s * 1e3) if prof_step_s > 0 else None,
            "other_bins_share_of_profiled_step": {b: round(bins[b][1] / (prof_step_s * 1e3), 4)
                                                  for b in bins if b != dom and bins[b][0] and prof_step_s > 0},
            # the other SpMM families beside the roofline kernel: algorithmic GB/s over their summed
            # launch times (the nodal bin spans many small, mostly L2-resident launch shapes)
            "other_bins": {b: {"launches": bins[b][0], "avg_launch_us": round(1e3 * bins[b][1] / bins[b][0], 2),
                               "achieved_gbs": round(bins[b][2] / (bins[b][1] * 1e-3) / 1e9, 1),
                               "frac": round(bins[b][2] / (bins[b][1] * 1e-3) / 1e9 / peak, 4)}
                           for b in bins if b != dom and bins[b][0] and bins[b][1] > 0}}

    # ---- e2e through the host-buffer C ABI ----------------------------------
    e2e = None
    log("e2e")
    if not args.no_e2e:
        h_x = np.zeros((ne, K), dtype=np.complex128)
        torch.cuda.synchronize()
        barrier(world)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            ctx.assemble_matrix(0)
            h_rhs = cols.assemble_host(ctx, rhs)
            h_x, _ = ctx.solve_block(colf, h_rhs, rtol=1e-8, max_it=200, inner_fp32=True)
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(time.perf_counter() - w0, world)
        nbytes = ne * K * 16
        e2e = {"value": world * K * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": 2 * nbytes,
               "path": "right-hand sides to the host (emg_assemble_rhs_mt_block, or the CSEM block kernel and a "
                       "D2H copy) + emg_solve_block (H2D rhs, D2H x), host wall clock"}

    # ---- plain FP64 drop-in on a subset of the columns ----------------------
    plain = None
    plain_fields = {}
    log("plain FP64 path")
    if single and args.plain_freqs != 0:
        npf = freqs.size if args.plain_freqs < 0 else min(args.plain_freqs, freqs.size)
        idx = np.unique(np.linspace(0, freqs.size - 1, npf).round().astype(int))
        # CSEM sweeps: at most --plain-tx transmitters per frequency
        txs = sorted(set(cols.src.tolist()))
        if cols.kind == "csem":
            txs = txs[::max(1, len(txs) // max(1, args.plain_tx))][:max(1, args.plain_tx)]
        loc = ctx if cols.kind == "csem" else None
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        p_info = []
        t_fields = 0.0

        def keep_fields(target, fi, j):
            # receiver fields of this solution for the accuracy report (not timed)
            nonlocal t_fields
            tf = time.perf_counter()
            if (rx_tets >= 0).all():
                plain_fields[j] = ctx.interpolate_fields(target, int(fi), rx, rx_tets)
            t_fields += time.perf_counter() - tf

        for fi in idx:
            ctx.assemble_matrix(int(fi))
            ctx.create_pc()
            if cols.kind == "mt":
                for mi, mode in enumerate((E.XY_POLAR, E.YX_POLAR)):
                    sr, si = ctx.assemble_rhs_mt(int(fi), mode)
                    inf = ctx.solve_linear_system(mode, sr, si, 300, 1e-8, raise_on_diverge=False)
                    p_info.append(inf.as_dict())
                    keep_fields(mode, fi, 2 * int(fi) + mi)
            else:
                for t in txs:
                    tx = np.asarray(prob.survey.tx[t], dtype=np.float64)
                    sr, si = ctx.assemble_rhs_csem(int(fi), tx, loc.find_cell_around_point(tx[None, :3]))
                    inf = ctx.solve_linear_system(E.SOL_CSEM, sr, si, 300, 1e-8, raise_on_diverge=False)
                    p_info.append(inf.as_dict())
                    keep_fields(E.SOL_CSEM, fi, int(fi) * len(prob.survey.tx) + int(t))
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - w0 - t_fields
        n_plain = len(p_info)
        plain = {"value": n_plain / t_plain, "unit": UNIT, "rhs": n_plain, "freqs": [float(freqs[i]) for i in idx],
                 "outer_its": [p["outer_its"] for p in p_info], "inner_its": [p["inner_its"] for p in p_info],
                 "true_rel_res": [p["true_rel_res"] for p in p_info],
                 "timing": "host wall clock around assemble_matrix + create_pc + (rhs + solve) per column, per "
                           "frequency"}

    # ---- accuracy of the headline solution against an FP64 solve ------------
    accuracy = None
    if single and not args.no_accuracy and (rx_tets >= 0).all():
        log("FP64 reference solve")
        x64 = torch.zeros_like(x)
        inf64 = ctx.solve_block_dev(colf, rhs.data_ptr(), x64.data_ptr(), rtol=1e-12, max_it=800,
                                    inner_fp32=False)
        accuracy = field_accuracy(ctx, E, cols, x, x64, rx, rx_tets, plain_fields)
        accuracy["reference"] = ("FP64 block solve of the same %d columns (FP64 FGMRES, FP64 FCG, FP64 AMS) "
                                 "to relative residual 1e-12" % K)
        accuracy["reference_true_rel_res_max"] = max(i.true_rel_res for i in inf64)
        log("accuracy: %s" % {k: accuracy[k] for k in ("E_max_rel", "H_max_rel", "rho_a_max_rel", "phase_max_deg")})
        del x64

    # ---- CPU baseline --------------------------------------------------------
    cpu = None
    log("cpu baseline")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            s = cpu_sample(prob)
            cal = cpu_calibration(args.config)
            if cal:
                inner, src = cal["inner_per_rhs"], "committed full oracle solves of this workload"
            elif plain:
                inner, src = float(np.mean(plain["inner_its"])) / 2.0, "GPU plain path inner counts"
            else:
                inner, src = 30 * s["inner"], "30 x sampled"
            v, per_rhs = cpu_rhs_per_s(s, inner)
            cpu = {"value": v, "unit": UNIT, "cores": s["threads"], "kind": "port",
                   "sample": ("CPU oracle on one frequency of this workload: assembly %.2fs, AMS setup %.2fs, "
                              "MT RHS %.2fs, %d FGMRES iteration(s) with %d inner FCG iterations in %.2fs; "
                              "RHS/s = 1/((asm+setup)/2 + rhs + %.1f inner its per RHS (%s) x time per inner "
                              "iteration)" % (s["t_asm"], s["t_setup"], s["t_rhs"], s["outer"], s["inner"],
                                              s["t_fgmres"], inner, src))}
        except Exception as ex:  # the baseline must not kill the benchmark line
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": "failed: %s" % ex}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 outer / f32 AMS (f64 AMS below %g Hz)" % ctx.get_option(
                "emg_block_fp64_below"), "data": "synthetic",
            "config": {"workload": prob.name, "tets": prob.mesh.n_tets, "edges": prob.mesh.n_edges,
                       "nnz": int(ctx.make_sparsity_patterns()[0][-1]), "rhs_per_step": K, "freqs_hz":
                       [float(f) for f in freqs], "rtol": 1e-8, "inner": "FCG(FP64) + AMS(FP32)",
                       "accuracy_policy": {
                           "fp32_columns_rtol": 1e-8 * ctx.get_option("emg_block_fp32_rtol_factor"),
                           "fp64_ams_below_hz": ctx.get_option("emg_block_fp64_below"),
                           "divergence_correction": bool(ctx.get_option("emg_div_correction")),
                           "why": "one relative residual leaves different receiver errors for different "
                                  "preconditioners: the FP32-preconditioned block columns iterate to rtol x 0.01 so "
                                  "that their receiver fields are as accurate as the per-RHS FP64 method's at rtol "
                                  "(field_err_vs_fp64)"},
                       "edge_smoother": "Chebyshev degree %d, %d sweep(s) per smoothing step" % (
                           ctx.get_option("emg_block_cheb_degree"), ctx.get_option("emg_block_relax_times")),
                       "warm_start": "none (zero guess)", "l2": "inputs larger than L2 (operator ~%.0f MB)" %
                       (int(ctx.make_sparsity_patterns()[0][-1]) * 20 / 1e6), "parallelism": "replicas" if world > 1 else "1 GPU",
                       "options": args.options or None},
            "e2e": e2e, "plain_fp64": plain, "field_err_vs_fp64": accuracy, "dual": dual, "warm_start": warm,
            "speedup_vs_plain_fp64": (value / world) / plain["value"] if plain else None,
            "converged": all_conv, "true_rel_res_max": max(c[0] for c in conv) if conv else None,
            "outer_its": [c[1] for c in conv],
            "roofline": roof if n_l else None, "profile_bins": {k: {"launches": v[0], "ms": v[1], "bytes": v[2]} for k, v in bins.items()},
            "phases_one_step": phases, "spmm_layouts": E.spmm_layouts(),
            "host_breakdown_s_per_step": timed_breakdown,
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches, "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
        if args.breakdown:
            print("breakdown (s over %d steps): %s" % (args.steps, breakdown), file=sys.stderr)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
