#!/usr/bin/env python
"""Benchmark of the IM-SRG(2) engine on B200.

Default workload (--workload flow), the metric's own configuration: seconds
to a converged ground-state energy of the 2-D quantum dot with N=20
electrons in R=20 shells at hbar-omega=0.5 (420 spin-orbitals, 61,947,679
entries = 495.6 MB per operator).  Input: Coulomb TBMEs (v_int in
__float128, because the reference's real(8) sums lose every digit at R=20)
and Hartree-Fock on the host (not timed).  One step = one whole Magnus
IM-SRG(2) flow (first-order Magnus, Euler steps of 0.7, nested BCH series,
White generator) from the HF Hamiltonian resident in HBM to |MBPT2| <= 1e-9,
FP64 throughout, ladders only as the reference's run_magnus (--pandya adds
the particle-hole channel).  value: seconds per converged E_gs (lower is
better); e2e: the same through the C ABI with the Hamiltonian uploaded from
pinned host memory and the evolved one downloaded every step.

--workload commutator: one FP64 commutator [Omega, H] of seeded random
operators at N=20, R=20 with the Pandya channel, in TFLOP/s of the reference
algorithm's FP64 work.

--workload batch: the N x hbar-omega grid of 16 flows, concurrently
(qd_magnus_flow_batch) and one after another.

--gpus N (under torchrun): N independent replicas, one per GPU, no data-path
collective (weak scaling); the timed region is bracketed by barriers and the
max over ranks is reported.

--impl reference: the CPU restatement of the reference (oracle/, OpenMP,
OpenBLAS dgemm) on the host cores, loading no product library, on a bounded
sample of the same workload: per step one block-sampled phase of the flow's
commutator (phases rotate, covering whole commutators), scaled to one flow
by the FP64 flow's commutator count; or of the random commutator.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to converged E_gs (N=20,R=20, |dE|<=1e-6): chosen form vs FP64 GPU; TFLOP/s"
NBODY, EMAX = 20, 20
SEED_H, SEED_OMEGA = 1, 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nbody", type=int, default=NBODY)
    ap.add_argument("--emax", type=int, default=EMAX)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graphs", action="store_true",
                    help="flow: launch every kernel eagerly (a profiler then lists every launch)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--ref-stride", type=int, default=8)
    ap.add_argument("--batch-max-iter", type=int, default=300, help="batch: flow step limit per instance")
    ap.add_argument("--ws-train", type=int, default=64, help="warmstart: training draws")
    ap.add_argument("--ws-eval", type=int, default=16, help="warmstart: held-out draws at N=20, R=20")
    ap.add_argument("--ws-steps", type=int, default=3000, help="warmstart: Adam steps")
    ap.add_argument("--ws-sample", type=int, default=4096, help="warmstart: recorded entries per flow")
    ap.add_argument("--ws-eval-seed", type=int, default=77, help="warmstart: seed of the held-out draws")
    ap.add_argument("--ws-frac", default="0.5,0.7,0.85",
                    help="warmstart: target s as fractions of the training flows' median final s; the first "
                         "is the headline, the others are reported beside it")
    ap.add_argument("--workload", choices=["flow", "commutator", "batch", "warmstart"], default="flow")
    ap.add_argument("--split", type=int, default=0,
                    help="flow/commutator: block contractions in the split form with this many BF16 slices "
                         "(0 = plain FP64)")
    ap.add_argument("--hw", type=float, default=0.5)
    ap.add_argument("--pandya", action="store_true", help="flow: add the particle-hole channel")
    ap.add_argument("--hf-mix", type=float, default=0.5, help="flow: HF density mixing (1 = plain iteration)")
    ap.add_argument("--tbme", choices=["quad", "reference"], default="quad",
                    help="flow: v_int in __float128 (quad) or in the reference's real(8) sums")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# --------------------------------------------------------------------------
# nvidia-smi clock sampler (started before, stopped after the timed region)
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = str(local_rank)
        if vis:
            parts = [p.strip() for p in vis.split(",") if p.strip()]
            if local_rank < len(parts) and parts[local_rank].isdigit():
                idx = parts[local_rank]
        self.idx = idx
        self.proc = None
        self.path = os.path.join("/tmp", "qd_clocks_%d_%d.csv" % (os.getpid(), local_rank))

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.idx, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


# --------------------------------------------------------------------------
def measured_dgemm_tflops(torch, device) -> float:
    """cuBLAS DGEMM throughput (8192^3, best of 3) as the FP64 tensor-pipe peak."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize(device)
    best = 1e30
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def stage_roofline(prof: dict, flops: dict, neq2b: int, dgemm_peak: float, hbm_peak: float, split: int = 0) -> dict:
    """Roofline of the stage with the largest device time."""
    name, (ms, cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    per_launch_s = (ms / max(cnt, 1)) / 1e3
    if split and name in ("ladder_gemm", "pandya_gemm"):
        # the split form runs slice_pairs(split) BF16 products per FP64 product
        f = flops["ladder"] if name == "ladder_gemm" else flops["pandya"] / 2
        return {"kernel": "k_split_gemm (%s, %d slices)" % (name, split), "bound": "tensor",
                "achieved": f * slice_pairs(split) / per_launch_s / 1e12, "peak": bf16_peak_tflops(),
                "unit": "TFLOP/s", "peak_source": bf16_source(),
                "algorithmic_per_launch": f * slice_pairs(split),
                "note": "BF16 slice-product FLOPs = FP64-algorithm FLOPs x %d slice pairs; the stage time "
                        "includes slicing the operands" % slice_pairs(split)}
    if name == "ladder_gemm":
        return {"kernel": "k_grouped_gemm (ladders of commutator_222)", "bound": "tensor",
                "achieved": flops["ladder"] / per_launch_s / 1e12, "peak": dgemm_peak, "unit": "TFLOP/s",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64; tcgen05 has no f64 kind)",
                "algorithmic_per_launch": flops["ladder"]}
    if name == "pandya_gemm":
        # one r x r x nb product per cross-coupled block (the reference does two)
        return {"kernel": "k_grouped_gemm (Pandya products)", "bound": "tensor",
                "achieved": flops["pandya"] / 2 / per_launch_s / 1e12, "peak": dgemm_peak, "unit": "TFLOP/s",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                "algorithmic_per_launch": flops["pandya"] / 2}
    if name == "c122":
        byts = 3.0 * 8 * neq2b  # read A, B two-body, write C two-body
        return {"kernel": "k_122 (commutator_122)", "bound": "hbm", "achieved": byts / per_launch_s / 1e9,
                "peak": hbm_peak, "unit": "GB/s", "peak_source": hbm_source(),
                "algorithmic_per_launch": byts}
    byts = 3.0 * 8 * neq2b
    return {"kernel": name, "bound": "hbm", "achieved": byts / per_launch_s / 1e9, "peak": hbm_peak,
            "unit": "GB/s", "peak_source": hbm_source(), "algorithmic_per_launch": byts}


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# engine's stages, from one ncu capture of the N=20, R=17 case (19,841,598
# entries per operator, inputs above L2).  GEMM and gather traffic is operand
# and output traffic, so it is scaled to the benchmarked basis by the number
# of entries per operator.
NCU_NEQ = 19841598
NCU_TRAFFIC = {"ladder_gemm": 794.761728e6 + 162.643712e6, "pandya_gemm": 200.469760e6 + 676.389888e6,
               "pandya_gather": 2126.409e6 + 154.573824e6}
# commutator_122 of one flow commutator [Omega, X] (the k_122_pppp and
# k_122_gen launches), from the N=20, R=18 capture (29,618,726 entries per
# operator): scaled to the flow's basis by entries per operator
NCU_FLOW_NEQ = 29618726
NCU_FLOW_TRAFFIC = {"c122": (29.3e6 + 139.6e6) + (179.3e6 + 51.9e6)}


def _peaks_present() -> bool:
    return os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json"))


def hbm_source() -> str:
    return ("MEASURED_PEAKS.json hbm_gbs (of measured)" if _peaks_present()
            else "fallback 6650 GB/s: MEASURED_PEAKS.json absent (of fallback)")


def bf16_source() -> str:
    return ("MEASURED_PEAKS.json bf16_tflops (of measured, burst)" if _peaks_present()
            else "fallback 1590 TFLOP/s: MEASURED_PEAKS.json absent (of fallback)")


def hbm_peak_gbs() -> float:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"])
    except Exception:
        return 6650.0


def bf16_peak_tflops() -> float:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["bf16_tflops"])
    except Exception:
        return 1590.0


def form_name(split: int) -> str:
    return ("split: block contractions as %d BF16 slices per operand (tcgen05, exact FP32 chunks, FP64 sum)"
            % split) if split else "plain FP64"


def slice_pairs(split: int) -> int:
    return split * (split + 1) // 2


def cpu_baseline_full(a: np.ndarray, b: np.ndarray, flops_total: float) -> dict:
    """The oracle on the host cores: one complete [Omega,H] (N=20,R=20, Pandya
    channel on), phases of the block sampler run back to back."""
    import oracle

    O = oracle.Layout(NBODY, EMAX)
    A, B, Cop = oracle.Op(O, -1, a), oracle.Op(O, 1, b), oracle.Op(O, 1)
    S = oracle.Sampler(A)
    stride = 4
    t0 = time.perf_counter()
    for ph in range(stride):
        S.run(A, B, Cop, stride, ph)
    dt = time.perf_counter() - t0
    return {"value": flops_total / dt / 1e12, "unit": "TFLOP/s", "cores": oracle.get_threads(), "kind": "port",
            "seconds": dt, "blas": os.path.basename(oracle.BLAS) if oracle.BLAS else "oracle loop dgemm",
            "sample": "one complete [Omega,H] at N=20,R=20 with the Pandya channel, same inputs "
                      "(oracle restatement, OpenMP over blocks, OpenBLAS dgemm)"}


# --------------------------------------------------------------------------
class _OracleLayoutView:
    """The attributes qd_imsrg_b200.flops reads, from an oracle.Layout (the
    reference arm loads no product library)."""

    def __init__(self, O):
        self.nbody, self.msp, self.nblock, self.dims, self.emax = O.n, O.m, O.nblock, O.dims, O.emax
        self.ccn, self.cc_r, self.cc_nb = O.ccn, O.cc_r, O.cc_nb


def oracle_operator(O, herm: int, rng, parts=None, sigma: float = 0.1) -> np.ndarray:
    """Seeded operator in vectorize order for an oracle.Layout, generated with
    numpy: entries N(0, sigma^2), diagonal-class blocks (fhh, fpp, Vhhhh,
    Vpppp, Vphph) made (X + herm X^T)/2, one-body entries that change (m_l, m_s)
    zeroed, E0 = 0.  parts: names of the parts kept non-zero (default all)."""
    v = rng.normal(0.0, sigma, O.neq)
    v[0] = 0.0
    n, m = O.n, O.m
    mp = m - n
    g = O.qn[:, 1] * 10 + O.qn[:, 2]
    keep = set(parts) if parts is not None else None

    def put(name, o, rows, cols, sym, gr=None, gc=None):
        X = v[o:o + rows * cols].reshape(rows, cols, order="F")
        if keep is not None and name not in keep:
            X[:] = 0.0
        else:
            if sym:
                X[:] = (X + herm * X.T) / 2
            if gr is not None:
                X[gr[:, None] != gc[None, :]] = 0.0
        v[o:o + rows * cols] = X.reshape(-1, order="F")

    o = 1
    put("fhh", o, n, n, True, g[:n], g[:n]); o += n * n
    put("fpp", o, mp, mp, True, g[n:], g[n:]); o += mp * mp
    put("fph", o, mp, n, False, g[n:], g[:n])
    names = ["Vhhhh", "Vpppp", "Vpphh", "Vphph", "Vppph", "Vphhh"]
    for q in range(O.nblock):
        nh, nb, npp = (int(x) for x in O.dims[q, :3])
        shapes = [(nh, nh, True), (npp, npp, True), (npp, nh, False), (nb, nb, True), (npp, nb, False),
                  (nb, nh, False)]
        for k, (r, c, sym) in enumerate(shapes):
            if r * c:
                put(names[k], int(O.offs[q, k]), r, c, sym)
    return v


def run_reference(args, world, rank):
    """Reference arm of the commutator workload: the oracle on the host
    cores, one block-sampled phase of [Omega, H] per step."""
    if rank != 0:
        return 0
    import oracle
    from qd_imsrg_b200.flops import commutator_flops

    O = oracle.Layout(args.nbody, args.emax)
    rng = np.random.default_rng(SEED_H)
    b = oracle_operator(O, 1, rng)
    a = oracle_operator(O, -1, rng)
    fl = sample_flops(_OracleLayoutView(O), args.ref_stride)
    A, B, Cop = oracle.Op(O, -1, a), oracle.Op(O, 1, b), oracle.Op(O, 1)
    S = oracle.Sampler(A)
    stride = args.ref_stride
    # phase 0 fills the cross-coupled matrices; warm-up starts there
    for w in range(args.warmup):
        S.run(A, B, Cop, stride, w % stride)
    done, t = 0.0, 0.0
    for k in range(args.steps):
        ph = (args.warmup + k) % stride
        if ph != 0 and k == 0:
            S.run(A, B, Cop, stride, 0)  # cross-coupled matrices for this run
        t0 = time.perf_counter()
        S.run(A, B, Cop, stride, ph)
        t += time.perf_counter() - t0
        done += fl[ph]
    val = done / t / 1e12
    total = commutator_flops(_OracleLayoutView(O))["total"]
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded numpy operators)",
            "config": {"workload": "FP64 [Omega,H] N=%d R=%d, Pandya on; reference arm: CPU restatement"
                                   % (args.nbody, args.emax), "block_stride": stride,
                       "flops_per_commutator": total},
            "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": oracle.get_threads(), "kind": "port",
                             "sample": "per step the two-body work of every %d-th (M_L,M_S) block and "
                                       "cross-coupled block (phase rotating; phase 0 adds E0 and the "
                                       "one-body parts), throughput = reference-algorithm FLOPs of the "
                                       "sample / time" % stride},
            "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def split_errors(P, got, ref) -> dict:
    """Relative Frobenius error per stored part (and E0) of a split-form
    result against the FP64 result of the same inputs."""
    n, mp = P.nbody, P.msp - P.nbody
    parts = {"E0": [np.array([0])]}
    o = 1
    for name, sz in (("fhh", n * n), ("fpp", mp * mp), ("fph", mp * n)):
        parts[name] = [np.arange(o, o + sz)]
        o += sz
    names = ["Vhhhh", "Vpppp", "Vpphh", "Vphph", "Vppph", "Vphhh"]
    for nm in names:
        parts[nm] = []
    for q in range(P.nblock):
        nh, nb, npp = (int(x) for x in P.dims[q, :3])
        for k, sz in enumerate((nh * nh, npp * npp, npp * nh, nb * nb, npp * nb, nb * nh)):
            if sz:
                st = int(P.offs[q, k])
                parts[names[k]].append(np.arange(st, st + sz))
    out = {}
    for nm, ix in parts.items():
        if not ix:
            continue
        ix = np.concatenate(ix)
        d = np.linalg.norm(got[ix] - ref[ix])
        r = np.linalg.norm(ref[ix])
        out[nm] = float(d / r) if r > 0 else float(d)
    out["max"] = max(out.values())
    return out


def sample_flops(P, stride):
    """Reference-algorithm FLOPs done by each phase of the block sampler."""
    from qd_imsrg_b200.flops import commutator_flops_parts

    parts = commutator_flops_parts(P)
    out = []
    for ph in range(stride):
        f = parts["block"][ph::stride].sum() + parts["cc"][ph::stride].sum()
        if ph == 0:
            f += parts["onebody"]
        out.append(float(f))
    return out


# --------------------------------------------------------------------------
# Commutators of the converged FP64 flow at the benchmarked configurations
# (the flow is deterministic: every run takes the same steps).  They scale
# the CPU restatement's time per commutator to seconds per E_gs where the
# whole CPU flow would take hours.
FLOW_COMMUTATORS = {(20, 20, 0.5, False): 181, (20, 20, 0.5, True): 115}


def flow_input(args, nbody=None, emax=None, hw=None):
    """HF Hamiltonian of a flow workload (host, not timed)."""
    import qd_imsrg_b200 as qd

    t0 = time.perf_counter()
    vec, eig, hf_it = qd.hf_hamiltonian(nbody or args.nbody, emax or args.emax, hw or args.hw, mix=args.hf_mix,
                                        quad=args.tbme == "quad")
    return vec, eig, hf_it, time.perf_counter() - t0


def cpu_flow_estimate(vec, eig, args, commutators: int) -> dict:
    """The oracle on the host cores on one whole commutator of the flow: the
    flow's first BCH commutator [Omega, H], Omega = 0.7 eta(H_HF), run as the
    `ref_stride` block-sampled phases back to back (together exactly one
    commutator); seconds per E_gs = its time times the flow's commutator
    count (an extrapolation: the whole CPU flow would take about an hour)."""
    import oracle

    O = oracle.Layout(args.nbody, args.emax, eig=eig)
    H = oracle.Op(O, 1, vec)
    eta = oracle.Op(O, -1)
    oracle.build_white(eta, H)
    G = oracle.Op(O, -1)
    oracle.add_arrays(G, 1.0, eta, float(np.float32(0.7)), G)
    C = oracle.Op(O, 1)
    S = oracle.Sampler(G)
    stride = args.ref_stride
    t0 = time.perf_counter()
    for ph in range(stride):
        S.run(G, H, C, stride, ph, pandya=args.pandya)
    per_comm = time.perf_counter() - t0
    return {"value": per_comm * commutators, "unit": "s per converged E_gs", "cores": oracle.get_threads(),
            "kind": "port", "seconds_per_commutator": per_comm, "commutators": commutators,
            "sample": "one whole commutator [Omega, H] of the flow (Omega = 0.7 eta(H_HF), its %d block "
                      "phases back to back) timed on the oracle (OpenMP, OpenBLAS); seconds per E_gs "
                      "extrapolated: that time x the %d commutators of this run's FP64 GPU flow" %
                      (stride, commutators)}


def flow_desc(args):
    return "Magnus IM-SRG(2) flow to |MBPT2| <= 1e-9, N=%d R=%d hbar-omega=%g, %s" % (
        args.nbody, args.emax, args.hw, "particle-hole channel on" if args.pandya else "ladders only (run_magnus)")


def run_flow(args, world, rank, local):
    """Seconds to a converged ground-state energy: Hartree-Fock on the host,
    then the Magnus flow on the device to |MBPT2(H(s))| <= 1e-9, one flow per
    step."""
    import torch

    import qd_imsrg_b200 as qd

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    vec, eig, hf_it, setup_s = flow_input(args)
    P = qd.Layout(args.nbody, args.emax, eig=eig, device=local)
    stream = torch.cuda.Stream(device=device)
    P.set_stream(stream.cuda_stream)
    if args.no_graphs:
        P.set_graphs(False)
    H, HS = qd.FullHam(P, 1, vec), qd.FullHam(P, 1)

    def flow():
        return qd.magnus_flow(H, HS, pandya=args.pandya, max_iter=1000)

    fp64 = None
    if args.split:
        # the plain FP64 flow on the same Hamiltonian, for the error of the split form
        _, r0 = flow()
        fp64 = {"E_gs": float(r0.E0), "flow_steps": int(r0.iterations), "commutators": int(r0.commutators)}
        P.split = args.split

    for _ in range(max(1, args.warmup)):
        tr, res = flow()
    clocks = ClockSampler(local)
    launches0 = P.launches()
    barrier(world)
    torch.cuda.synchronize(device)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        tr, res = flow()
    torch.cuda.synchronize(device)
    sec = (time.perf_counter() - t0) / args.steps
    clk = clocks.stop()
    barrier(world)
    launches = (P.launches() - launches0) // max(1, args.steps)
    sec = max_over_ranks(sec, world, device)
    # one more flow with the per-stage event profiler (outside the timed region)
    P.profile(True)
    flow()
    torch.cuda.synchronize(device)
    prof = P.profile_read()
    P.profile(False)
    # end to end: Hamiltonian uploaded from pinned host memory, evolved one downloaded, every step
    hv = torch.from_numpy(vec).pin_memory().numpy()
    hout = torch.empty(P.neq, dtype=torch.float64).pin_memory().numpy()
    ne2e = max(1, min(args.steps, args.e2e_steps))
    barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(ne2e):
        H.upload(hv)
        flow()
        hout[:] = HS.download()
    e2e_sec = max_over_ranks((time.perf_counter() - t0) / ne2e, world, device)
    comms = int(res.commutators)
    n, mp = P.nbody, P.msp - P.nbody
    neq2b = P.neq - (1 + n * n + mp * mp + mp * n)
    name, (ms, cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    per = (ms / max(cnt, 1)) / 1e3
    byts = 3.0 * 8 * neq2b
    roof = {"kernel": name, "bound": "hbm", "achieved": byts / per / 1e9, "peak": hbm_peak_gbs(), "unit": "GB/s",
            "peak_source": hbm_source(), "algorithmic_per_launch": byts,
            "note": "stage with the most device time, per launch = per commutator; bytes = read A, B and "
                    "write C two-body parts once",
            "traffic": NCU_FLOW_TRAFFIC[name] * P.neq / NCU_FLOW_NEQ if name in NCU_FLOW_TRAFFIC else None,
            "traffic_source": "ncu dram bytes of the k_122_pppp and k_122_gen launches of one commutator at N=20 R=18, "
                              "scaled by entries per operator" if name in NCU_FLOW_TRAFFIC else None}
    roof["frac"] = roof["achieved"] / roof["peak"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_flow_estimate(vec, eig, args, comms)
    if rank == 0:
        line = {"metric": METRIC, "value": sec, "unit": "s per converged E_gs", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: Coulomb TBMEs from v_int and Hartree-Fock computed on the host",
                "config": {"workload": flow_desc(args), "form": form_name(args.split),
                           "cuda_graphs": not args.no_graphs,
                           "chosen_form": "plain FP64 block contractions, BCH terms replayed as CUDA graphs: on "
                                          "this ladders-only flow the split form (--split S) and the learned "
                                          "warm start (--workload warmstart) measure slower",
                           "E_HF": float(vec[0]),
                           "fp64_flow": fp64,
                           "dE_vs_fp64": (abs(float(res.E0) - fp64["E_gs"]) if fp64 else None),
                           "E_gs": float(res.E0), "flow_steps": int(res.iterations), "rejected": int(res.rejected),
                           "commutators": comms, "s_final": float(res.s), "hf_setup_s": setup_s,
                           "hf_iterations": hf_it, "hf_mix": args.hf_mix, "tbme": args.tbme,
                           "bch_terms": [int(x) for x in tr[:, 6]],
                           "l2": "every step streams 495.6 MB operators, far above the 126 MB L2",
                           "parallelism": "replicas x%d" % world},
                "e2e": {"value": e2e_sec, "unit": "s per converged E_gs", "h2d_bytes_per_step": 8 * P.neq,
                        "d2h_bytes_per_step": 8 * P.neq},
                "roofline": roof, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
                "stages_ms_per_flow": {k: v[0] for k, v in prof.items()}}
        print(json.dumps(line), flush=True)
    for o in (H, HS):
        o.close()
    P.close()
    return 0


# Batched instances: N x hbar-omega, R=16 for N <= 12 and R=20 otherwise
BATCH_GRID = [(nb, hw) for nb in (6, 12, 20, 30) for hw in (0.1, 0.28, 0.5, 1.0)]


def run_batch(args, world, rank, local):
    """16 independent flows (the N x hbar-omega grid) run concurrently by
    qd_magnus_flow_batch (one host thread and stream per instance) against
    the same flows one after another; per-instance E_gs must agree."""
    import torch

    import qd_imsrg_b200 as qd

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    inst, skipped = [], []
    for nb, hw in BATCH_GRID:
        R = 16 if nb <= 12 else 20
        try:
            vec, eig, _, _ = flow_input(args, nb, R, hw)
        except qd.QDError as e:
            skipped.append({"N": nb, "hw": hw, "R": R, "why": str(e)})
            continue
        P = qd.Layout(nb, R, eig=eig, device=local)
        inst.append({"N": nb, "hw": hw, "R": R, "P": P, "H": qd.FullHam(P, 1, vec), "HS": qd.FullHam(P, 1),
                     "E_HF": float(vec[0])})
    setup_s = time.perf_counter() - t0
    kw = dict(pandya=args.pandya, max_iter=args.batch_max_iter)
    # one after another (also allocates every layout's flow workspaces)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for d in inst:
        try:
            _, r = qd.magnus_flow(d["H"], d["HS"], **kw)
            d["E_sep"], d["steps"], d["ok"] = float(r.E0), int(r.iterations), True
        except qd.QDError as e:
            d["ok"], d["why"] = False, str(e)
    torch.cuda.synchronize(device)
    t_sep = time.perf_counter() - t0
    good = [d for d in inst if d["ok"]]
    pairs = [(d["H"], d["HS"]) for d in good]
    # the thread-per-instance stream mode, for comparison (outside the timed region)
    for _ in range(max(1, args.warmup - 1)):
        qd.magnus_flow_batch(pairs, raise_on_error=False, streams=True, **kw)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    res_s, st_s = qd.magnus_flow_batch(pairs, raise_on_error=False, streams=True, **kw)
    torch.cuda.synchronize(device)
    t_streams = time.perf_counter() - t0
    # lockstep: one launch per kernel over all instances' tiles (timed)
    for _ in range(max(0, args.warmup - 1)):
        qd.magnus_flow_batch(pairs, raise_on_error=False, **kw)
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize(device)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res, st = qd.magnus_flow_batch(pairs, raise_on_error=False, **kw)
    torch.cuda.synchronize(device)
    t_batch = (time.perf_counter() - t0) / args.steps
    clk = clocks.stop()
    t_batch = max_over_ranks(t_batch, world, device)
    worst = worst_s = 0.0
    for d, r, s_, rs in zip(good, res, st, res_s):
        d["E_batch"], d["status"] = float(r.E0), s_
        worst = max(worst, abs(d["E_batch"] - d["E_sep"]))
        worst_s = max(worst_s, abs(float(rs.E0) - d["E_sep"]))
    if rank == 0:
        per = [{k: d[k] for k in ("N", "hw", "R", "E_HF", "E_sep", "E_batch", "steps") if k in d} for d in good]
        fails = [{"N": d["N"], "hw": d["hw"], "R": d["R"], "why": d["why"]} for d in inst if not d["ok"]]
        line = {"metric": "s for the %d converged E_gs of the N x hbar-omega grid (batched flows)" % len(good),
                "value": t_batch, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * t_batch, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic: Coulomb TBMEs from v_int and Hartree-Fock computed on the host",
                "config": {"workload": "batched Magnus IM-SRG(2) flows, N in {6,12,20,30} x hbar-omega in "
                                       "{0.1,0.28,0.5,1.0}, R=16 for N<=12 else 20, %s; lockstep, each BCH "
                                       "term's 122 tiles and ladder tasks of all instances in one launch per "
                                       "kernel" % ("particle-hole channel on" if args.pandya else "ladders only"),
                           "separate_s": t_sep, "speedup_vs_separate": t_sep / t_batch,
                           "streams_s": t_streams, "speedup_vs_streams": t_streams / t_batch,
                           "max_abs_dE_batch_vs_separate": worst, "max_abs_dE_streams_vs_separate": worst_s,
                           "instances": per, "flow_failed": fails,
                           "hf_failed": skipped, "setup_s": setup_s},
                "clocks": clk}
        print(json.dumps(line), flush=True)
    for d in inst:
        d["H"].close()
        d["HS"].close()
        d["P"].close()
    return 0


def run_warmstart(args, world, rank, local):
    """Learned warm start: train the per-entry network on plain-flow Omega(s)
    trajectories (hbar-omega ~ U[0.1, 1], N in {12, 20}, R in {16, 20}), then
    on held-out hbar-omega at N=20, R=20 run the plain flow from Omega = 0
    (cold) and from the predicted Omega(s_target) (warm)."""
    import torch

    from qd_imsrg_b200 import warmstart as ws

    torch.cuda.set_device(local)
    rng = np.random.default_rng(2024)
    t0 = time.perf_counter()
    Xs, Ts, sfin, nsteps, trfail = [], [], {}, {}, []
    for k in range(args.ws_train):
        nb, R = (12, 20)[k % 2], (16, 20)[(k // 2) % 2]
        hw = float(rng.uniform(0.1, 1.0))
        try:
            inst = ws.Instance(nb, R, hw, device=local, mix=args.hf_mix, quad=args.tbme == "quad")
        except Exception as e:  # HF failure: the draw is dropped
            trfail.append({"N": nb, "R": R, "hw": hw, "why": str(e)})
            continue
        try:
            idx, svals, om, res = ws.trajectory(inst, args.ws_sample, rng)
            X, T = ws.samples(inst, idx, svals, om)
            Xs.append(X)
            Ts.append(T)
            sfin.setdefault((nb, R), []).append(float(res.s))
            nsteps.setdefault((nb, R), []).append(int(res.iterations))
        except Exception as e:
            trfail.append({"N": nb, "R": R, "hw": hw, "why": str(e)})
        inst.close()
        torch.cuda.empty_cache()
    X, T = torch.cat(Xs), torch.cat(Ts)
    t_data = time.perf_counter() - t0
    mlp = ws.MLP(local, seed=7)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = ws.train(mlp, X, T, steps=args.ws_steps, batch=8192, lr=1e-3, seed=1, log_every=max(1, args.ws_steps // 10))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    ref_s = sfin.get((20, 20)) or [v for vals in sfin.values() for v in vals] or [20.0]
    fracs = [float(x) for x in args.ws_frac.split(",")]
    s_targets = [f * float(np.median(ref_s)) for f in fracs]
    s_target = s_targets[0]

    evals = []
    erng = np.random.default_rng(args.ws_eval_seed)  # held-out draws: their own generator
    for k in range(args.ws_eval):
        hw = float(erng.uniform(0.1, 1.0))
        try:
            inst = ws.Instance(20, 20, hw, device=local, mix=args.hf_mix, quad=args.tbme == "quad")
        except Exception as e:
            evals.append({"hw": hw, "why": str(e)})
            continue
        try:
            # one untimed flow first: the layout's first flow builds its plans,
            # tunes commutator_122 and captures the BCH step graphs, which the
            # timed cold and warm flows then both find ready
            ws.cold_flow(inst)
            cold = ws.cold_flow(inst)
            warms = [ws.warm_flow(mlp, inst, st) for st in s_targets]
            evals.append({"hw": hw, "E_HF": inst.E_HF, "cold": cold, "warm": warms[0], "sweep": warms[1:],
                          "dE": abs(warms[0]["E"] - cold["E"])})
        except Exception as e:
            evals.append({"hw": hw, "why": str(e)})
        inst.close()
        torch.cuda.empty_cache()
    ok = [e for e in evals if "cold" in e]
    if rank == 0:
        tot = lambda key, side: sum(e[side][key] for e in ok)
        line = {"metric": "learned warm start: flow seconds, N=20 R=20, held-out hbar-omega (warm vs cold)",
                "value": tot("seconds", "warm") / max(1, len(ok)), "unit": "s per converged E_gs (warm start)",
                "n_gpus": world, "steps": len(ok), "warmup": 0, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 flow, bf16/f32 network",
                "data": "synthetic: Coulomb TBMEs and HF computed on the host; network trained on the plain "
                        "flow's own Omega(s) trajectories",
                "config": {"workload": "Magnus flows N=20 R=20 from Omega = 0 and from the network's "
                                       "Omega(s_target)", "s_target": s_target,
                           "cold_s_per_flow": tot("seconds", "cold") / max(1, len(ok)),
                           "speedup": tot("seconds", "cold") / max(1e-30, tot("seconds", "warm")),
                           "steps_cold": tot("steps", "cold"), "steps_warm": tot("steps", "warm"),
                           "commutators_cold": tot("commutators", "cold"),
                           "commutators_warm": tot("commutators", "warm"),
                           "accepted": sum(1 for e in ok if e["warm"]["accepted"]), "evaluated": len(ok),
                           "max_abs_dE": max([e["dE"] for e in ok] or [None]),
                           "s_fraction": fracs[0], "eval_seed": args.ws_eval_seed,
                           "sweep": [{"s_fraction": f, "s_target": st,
                                      "seconds_warm": sum(e["sweep"][k]["seconds"] for e in ok),
                                      "steps_warm": sum(e["sweep"][k]["steps"] for e in ok),
                                      "commutators_warm": sum(e["sweep"][k]["commutators"] for e in ok),
                                      "accepted": sum(1 for e in ok if e["sweep"][k]["accepted"]),
                                      "max_abs_dE": max(abs(e["sweep"][k]["E"] - e["cold"]["E"]) for e in ok)
                                      if ok else None}
                                     for k, (f, st) in enumerate(zip(fracs[1:], s_targets[1:]))],
                           "train_rows": int(X.shape[0]), "train_draws": len(Xs), "train_failed": trfail,
                           "data_s": t_data, "train_s": t_train, "loss_history": hist, "per_instance": evals}}
        print(json.dumps(line, default=float), flush=True)
    mlp.close()
    return 0


def run_reference_flow(args, world, rank):
    """Reference arm of the flow workload: the oracle (the CPU restatement of
    the reference) on the host cores, loading no product library.  One step
    = one block-sampled phase of the flow's commutator [Omega, H]; phases
    rotate, so the steps cover whole commutators.  Operands: seeded numpy
    operators with the zero-part pattern of the flow's commutators (Omega:
    fph and Vpphh only, the White generator's parts; H: every part).  The
    oracle's work is fixed by the block structure and by which parts are
    zero, not by the values, so this is the cost of the flow's commutator.
    Seconds per converged E_gs = seconds per commutator (the sum of the
    phases' mean times) x the FP64 flow's commutator count at this
    configuration (an extrapolation, labelled as such)."""
    if rank != 0:
        return 0
    import oracle

    key = (args.nbody, args.emax, args.hw, bool(args.pandya))
    comms = FLOW_COMMUTATORS.get(key)
    t_setup = time.perf_counter()
    O = oracle.Layout(args.nbody, args.emax)
    rng = np.random.default_rng(SEED_H)
    h = oracle_operator(O, 1, rng)
    g = oracle_operator(O, -1, rng, parts=("fph", "Vpphh"))
    G, H, Cop = oracle.Op(O, -1, g), oracle.Op(O, 1, h), oracle.Op(O, 1)
    del g, h
    S = oracle.Sampler(G)
    stride = args.ref_stride
    setup_s = time.perf_counter() - t_setup
    times = {}
    for k in range(args.warmup + args.steps):
        ph = k % stride
        t0 = time.perf_counter()
        S.run(G, H, Cop, stride, ph, pandya=args.pandya)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.setdefault(ph, []).append(dt)
    mean = {p: statistics.mean(v) for p, v in times.items()}
    covered = len(mean) == stride
    per_comm = sum(mean.values()) if covered else sum(mean.values()) * stride / max(1, len(mean))
    timed = sum(len(v) for v in times.values())
    ms_step = 1e3 * sum(sum(v) for v in times.values()) / max(1, timed)
    if comms is not None:
        val, unit = per_comm * comms, "s per converged E_gs"
        how = ("extrapolation: seconds per commutator x %d, the commutator count of the FP64 flow at this "
               "configuration (measured on the GPU engine, which matches the oracle flow's count at every "
               "size where both run)" % comms)
    else:
        val, unit, how = per_comm, "s per commutator", "no flow commutator count for this configuration"
    sample = ("per step one of the %d block-sampled phases of [Omega, H] (phases rotate; all %d timed %s), "
              "N=%d R=%d, seeded numpy operators with the flow's zero-part pattern; seconds per commutator = "
              "sum of the phases' mean times = %.3f s" % (stride, stride, "and averaged" if covered else
                                                          "not all covered: scaled by the phase count",
                                                          args.nbody, args.emax, per_comm))
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": unit, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded numpy operators with the zero-part pattern of the flow's commutators",
            "config": {"workload": flow_desc(args) + "; reference arm: CPU restatement (oracle), whole "
                                                     "commutators in rotating block phases",
                       "seconds_per_commutator": per_comm, "commutators": comms, "extrapolation": how,
                       "phases_covered": sorted(mean), "setup_s": setup_s},
            "cpu_baseline": {"value": val, "unit": unit, "cores": oracle.get_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.workload in ("flow", "batch", "warmstart") and args.impl == "ours":
        rc = {"flow": run_flow, "batch": run_batch, "warmstart": run_warmstart}[args.workload](args, world, rank, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc
    if args.impl == "reference":
        rc = run_reference_flow(args, world, rank) if args.workload == "flow" else run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc

    import torch

    import qd_imsrg_b200 as qd
    from qd_imsrg_b200.flops import commutator_flops

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    P = qd.Layout(args.nbody, args.emax, device=local)
    stream = torch.cuda.Stream(device=device)
    P.set_stream(stream.cuda_stream)
    fl = commutator_flops(P)
    neq = P.neq
    n, mp = P.nbody, P.msp - P.nbody
    neq2b = neq - (1 + n * n + mp * mp + mp * n)

    a = qd.random_operator(P, -1, SEED_OMEGA)
    b = qd.random_operator(P, 1, SEED_H)
    A, B, C = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
    err = None
    if args.split:
        # error of the split form against the plain FP64 engine on the same inputs
        qd.commutator(A, B, C, pandya=True)
        ref = C.download()
        P.split = args.split
        qd.commutator(A, B, C, pandya=True)
        got = C.download()
        err = split_errors(P, got, ref)
    P.split = args.split

    for _ in range(args.warmup):
        qd.commutator(A, B, C, pandya=True)
    P.synchronize()
    dgemm_peak = measured_dgemm_tflops(torch, device)

    clocks = ClockSampler(local)
    launches0 = P.launches()
    P.profile(True)
    barrier(world)
    torch.cuda.synchronize(device)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        qd.commutator(A, B, C, pandya=True)
    e1.record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    barrier(world)
    prof = P.profile_read()
    P.profile(False)
    launches = P.launches() - launches0
    sec = e0.elapsed_time(e1) / 1e3
    sec = max_over_ranks(sec, world, device)
    value = world * args.steps * fl["total"] / sec / 1e12

    # end to end through the public API with pinned host buffers
    ha = torch.from_numpy(a).pin_memory().numpy()
    hb = torch.from_numpy(b).pin_memory().numpy()
    hc = torch.empty(neq, dtype=torch.float64).pin_memory().numpy()
    import ctypes as _C

    from qd_imsrg_b200 import _native

    lib = _native.lib()
    barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        A.upload(ha)
        B.upload(hb)
        qd.commutator(A, B, C, pandya=True)
        _native.check(lib.qd_op_download(C.h, hc.ctypes.data_as(_C.POINTER(_C.c_double)), neq))
    e2e_sec = (time.perf_counter() - t0) / args.e2e_steps
    e2e_sec = max_over_ranks(e2e_sec, world, device)
    e2e = {"value": world * fl["total"] / e2e_sec / 1e12, "unit": "TFLOP/s",
           "h2d_bytes_per_step": 2 * 8 * neq, "d2h_bytes_per_step": 8 * neq, "ms_per_step": 1e3 * e2e_sec}

    roof = stage_roofline(prof, fl, neq2b, dgemm_peak, hbm_peak_gbs(), args.split)
    roof["frac"] = roof["achieved"] / roof["peak"]
    stage = max(prof.items(), key=lambda kv: kv[1][0])[0]
    roof["traffic"] = NCU_TRAFFIC[stage] * neq / NCU_NEQ if stage in NCU_TRAFFIC else None
    roof["traffic_source"] = ("ncu dram bytes of the N=20 R=17 capture, scaled by entries per operator"
                              if roof["traffic"] is not None else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.nbody == NBODY and args.emax == EMAX:
        cpu = cpu_baseline_full(a, b, fl["total"])

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox operators)",
            "config": {"workload": "FP64 commutator [Omega,H], N=%d R=%d (%d spin-orbitals), random "
                                   "(anti)Hermitian operators, Pandya channel on" % (n, P.emax, P.msp),
                       "form": form_name(args.split), "error_vs_fp64": err,
                       "n_electrons": n, "shells": P.emax, "neq_per_operator": neq,
                       "flops_per_step": fl["total"], "flops_breakdown": fl,
                       "l2": "inputs larger than L2 (two 495.6 MB operators read per step)",
                       "parallelism": "replicas x%d" % world},
            "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
            "stages_ms_per_step": {k: v[0] / args.steps for k, v in prof.items()},
            "dgemm_peak_tflops": dgemm_peak,
        }
        print(json.dumps(line), flush=True)
    # release device objects before the torch stream they run on goes away
    for o in (A, B, C):
        o.close()
    P.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
