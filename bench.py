#!/usr/bin/env python
"""Benchmark: RK4 site-updates/s of the 256^3 droplet quench (real-time LHY RK4).

Workload (precision config): LHY droplet, N = 5000, box [-L/2, L/2]^3 with L = 4 N^{1/3},
256^3 grid, cubic coefficient quenched to -3.3, quartic 5/2, real-time RK4, dt = 5e-5.
Start: Gaussian of width 0.5 N^{1/3} with seeded phase noise 1e-3 (synthetic, seed 2024);
the step's cost does not depend on the state.  One step = one full RK4 step (4 stages).

  value     site-updates/s, complex128, state resident in HBM (fields of 256 MiB >> L2, so
            no flush is needed between steps)
  fp32      the same in complex64 with FP64 reductions
  e2e       the same metric through the host-buffer entry point: every step uploads the
            state from pinned host memory, steps once, and downloads the result
  roofline  dominant kernel of the step, algorithmic bytes / CUDA-event duration

--impl reference times the CPU restatement of the reference's algorithm (oracle/, FFTs with
all host threads) on the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 256
N_ATOMS = 5000.0
DT = 5e-5
C3 = -3.3
C4 = 2.5
SEED = 2024

# algorithmic field transfers (read + write, units of one field) of each launch of an RK4
# step, in launch order.  Merged path (16 launches): per stage y-fwd, z (fwd * K^2 * inv),
# y-inv, x stage boundary (inverse x, stage epilogue, next stage prologue, forward x):
#   boundary 1->2: R W, psi        W k1, W                         4
#   boundary 2->3: R W, psi, k1    W k2, k1+2k2, W                 6
#   boundary 3->4: R W, psi, k2, a W k3, a+2k3, W                  7
#   boundary 4->1: R W, psi, k3, a W psi1, W                       6
# Five-pass path (20 launches): per stage x-fwd, y-fwd, z, y-inv, x-inv.
MERGED_BOUNDARY = [4, 6, 7, 6]
AXES_BOUNDARY = [4, 6, 7, 5]  # per-axis scheme: the boundary of stages 1-4 (Euler: 4)
STAGE_XFWD = [2, 3, 3, 3]
STAGE_XINV = [3, 5, 6, 5]
KIND_NAMES = {0: "x_fwd_prologue", 10: "y_fwd", 22: "z_fwd_kinetic_inv", 11: "y_inv", 1: "x_inv_epilogue",
              3: "x_stage_boundary", 12: "y_deriv", 2: "x_stage_boundary_axes"}


def workload_geometry():
    L = 4.0 * N_ATOMS ** (1.0 / 3.0)
    return (N_GRID,) * 3, (-L / 2,) * 3, (L / 2,) * 3


def initial_state():
    import numpy as np
    from numpy.random import default_rng

    shape, left, right = workload_geometry()
    # Gaussian of width 0.5 N^{1/3}, phase noise 1e-3, normalised to N (host, numpy only)
    sig = 0.5 * N_ATOMS ** (1.0 / 3.0)
    x = [left[d] + (right[d] - left[d]) / shape[d] * (np.arange(shape[d]) + 0.5) for d in range(3)]
    g = [np.exp(-xi * xi / (2 * sig * sig)) for xi in x]
    psi = (g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :]).astype(np.complex128)
    rng = default_rng(SEED)
    psi *= np.exp(1j * 1e-3 * rng.uniform(-1, 1, psi.shape))
    dV = 1.0
    for d in range(3):
        dV *= (right[d] - left[d]) / shape[d]
    psi *= math.sqrt(N_ATOMS / (float(np.sum(np.abs(psi) ** 2)) * dV))
    return np.asfortranarray(psi[..., None])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        # samples under load only (the sampler also runs a second before the timed region)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                if float(parts[7]) < 50:  # idle sample (before or after the timed region)
                    continue
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kind_name: str, dtype: str):
    """Per-launch DRAM bytes (read + write) of a kernel kind from the committed ncu summary of
    the same workload and precision, if one exists."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        v = d.get(dtype, {}).get(kind_name)
        if isinstance(v, dict):
            return v.get("bytes_per_launch_256cubed")
    return None


def _reduce(x: float, world: int, op: str) -> float:
    """x reduced over the ranks of the default process group (MAX or SUM); a CPU tensor under
    gloo, a CUDA tensor under NCCL.  Every rank must call it, in the same order."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    return _reduce(x, world, "max")


def sum_over_ranks(x: float, world: int) -> float:
    return _reduce(x, world, "sum")


def timed_repeats(run, stream, world: int, min_seconds: float):
    """Times `run` (exactly K steps) with CUDA events on `stream`, each repeat bracketed by a
    barrier and a device synchronisation on both sides, the max over ranks per repeat; repeats
    until `min_seconds` of timed work have passed (every rank runs the same count), so that the
    clock sampler sees the timed region.  Returns the per-repeat milliseconds."""
    import torch

    out = []
    reps = None
    while reps is None or len(out) < reps:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        out.append(ms)
        if reps is None:
            # one count for all ranks (ms is already the max over ranks)
            reps = max(1, min(1000, int(math.ceil(min_seconds * 1e3 / max(ms, 1e-3)))))
    return out


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    from gp5_b200 import _abi

    torch.cuda.set_device(local_rank)
    dev = local_rank
    shape, left, right = workload_geometry()
    psi0 = initial_state()
    sites = N_GRID ** 3
    stream = torch.cuda.Stream(device=dev)
    results = {}
    launches = 0
    # complex128; complex64 as created (stochastically rounded state update); complex64 with the
    # compensated update; complex64 rounded to nearest
    for key, prec, form in ((0, _abi.GP5_C128, ""), (1, _abi.GP5_C64, ""), (2, _abi.GP5_C64, "comp"),
                            (3, _abi.GP5_C64, "rn")):
        plan = _abi.Plan(shape, left, right, precision=prec, device=dev)
        plan.set_stream(stream.cuda_stream)
        func = _abi.Functional(plan, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
        st = _abi.Stepper(func, DT, _abi.GP5_STEP_RK4, imaginary=False)
        if form == "comp":
            st.set_compensation(True)
        elif form == "rn":
            st.set_stochastic_rounding(False)
        f = plan.field(psi0)
        st.advance(f, args.warmup)  # builds the step graph; W untimed steps
        with torch.cuda.stream(stream):
            with ClockSampler(dev) as clk:
                time.sleep(1.0)  # nvidia-smi is sampling before the timed region starts
                reps_ms = timed_repeats(lambda: st.advance(f, args.steps), stream, world, args.min_seconds)
            ms = statistics.median(reps_ms)
        lps = st.launches_per_step
        launches += (lps * args.steps + 1) * len(reps_ms)  # + the prologue transform of each advance call
        r = {"ms": ms, "ms_per_step": ms / args.steps, "value": world * sites * args.steps / (ms / 1e3),
             "clocks": clk.summary(), "launches_per_step": lps, "tiles": plan.tiles(),
             "repeats": len(reps_ms), "ms_per_step_spread": [min(reps_ms) / args.steps, max(reps_ms) / args.steps]}
        # per-launch durations of one step (CUDA events between launches, same stream)
        prof = st.profile(f, nrep=3)
        r["profile"] = prof
        if prec == _abi.GP5_C128:
            # end to end: pinned host state in, one step, result back, per step
            host_in = torch.empty(plan.field_bytes, dtype=torch.uint8).pin_memory()
            host_out = torch.empty(plan.field_bytes, dtype=torch.uint8).pin_memory()
            host_in.numpy()[:] = np.frombuffer(np.asfortranarray(psi0).tobytes(order="F"), dtype=np.uint8)
            host_out2 = torch.empty(plan.field_bytes, dtype=torch.uint8).pin_memory()
            n_e2e = max(3, min(args.steps, 20))
            st.advance_host(host_in.numpy(), host_out.numpy(), 1)  # warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                # one state at a time: upload, one step, download, in order
                torch.cuda.synchronize()
                if world > 1:
                    torch.distributed.barrier()
                e0.record(stream)
                for _ in range(n_e2e):
                    st.advance_host(host_in.numpy(), host_out.numpy(), 1)
                e1.record(stream)
                torch.cuda.synchronize()
                ems1 = max_over_ranks(e0.elapsed_time(e1), world)
                # the pipelined entry point: every step is a host state uploaded, stepped once
                # and downloaded, with the copies of neighbouring states overlapping the steps
                ins = [host_in.data_ptr()] * n_e2e
                outs = [(host_out if k % 2 == 0 else host_out2).data_ptr() for k in range(n_e2e)]
                st.advance_host_many(ins[:3], outs[:3], 1)  # warm (captures the device states' graphs)
                torch.cuda.synchronize()
                if world > 1:
                    torch.distributed.barrier()
                # e0 orders the first upload (the upload stream waits for the plan stream); the
                # call returns after the last download, so e1 is recorded after all copies
                e0.record(stream)
                st.advance_host_many(ins, outs, 1)
                e1.record(stream)
                torch.cuda.synchronize()
                ems = max_over_ranks(e0.elapsed_time(e1), world)
            launches += (lps + 1) * n_e2e * 2
            r["e2e"] = {"value": world * sites * n_e2e / (ems / 1e3), "unit": "site-updates/s",
                        "h2d_bytes_per_step": plan.field_bytes, "d2h_bytes_per_step": plan.field_bytes,
                        "steps": n_e2e, "ms_per_step": ems / n_e2e,
                        "entry_point": "gp5cu_stepper_advance_host_many (pinned host states, copies overlapping "
                                       "the steps of neighbouring states)",
                        "one_state_at_a_time": {"value": world * sites * n_e2e / (ems1 / 1e3),
                                                "ms_per_step": ems1 / n_e2e,
                                                "entry_point": "gp5cu_stepper_advance_host"}}
            r["field_bytes"] = plan.field_bytes
        results[key] = r
        del f, st, func, plan
        torch.cuda.synchronize()
    return results, launches


def cufft_comparator(dev: int, steps: int = 10, warmup: int = 3) -> dict:
    """cuFFT, through torch.fft, as a timed comparator (never the product path).

    On the bench workload, per precision: (1) one 3D forward + inverse transform pair of the
    256^3 field by cuFFT against gp5cu_fft's pair; (2) the product's RK4 step (stepper.cpp:46-71
    with the LHY functional, functional.cpp:105-122, and the laplacian of operators.cpp:28-36)
    written as unfused torch operations around cuFFT, timed per step, with its one-step
    difference from the product's step (relative to max |psi|).  CUDA events on the stream the
    work is queued on; inputs larger than L2."""
    import numpy as np
    import torch

    from gp5_b200 import _abi

    shape, left, right = workload_geometry()
    n = shape[0]
    L = right[0] - left[0]
    psi0 = initial_state()
    stream = torch.cuda.Stream(device=dev)
    out = {"note": "library comparator: cuFFT via torch.fft plus unfused torch element-wise kernels",
           "steps": steps}

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for key, prec, cdt, rdt in (("c128", _abi.GP5_C128, torch.complex128, torch.float64),
                                ("c64", _abi.GP5_C64, torch.complex64, torch.float32)):
        with torch.cuda.stream(stream):
            # the field's x-fastest layout is a C-order (z, y, x) tensor
            x0 = torch.from_numpy(np.ascontiguousarray(psi0[..., 0].transpose(2, 1, 0))).to(dev).to(cdt)
            m = torch.fft.fftfreq(n, d=1.0 / n, dtype=torch.float64, device=f"cuda:{dev}")
            k2 = ((2 * math.pi / L) * m) ** 2
            K2 = ((k2[None, None, :] + k2[None, :, None]) + k2[:, None, None]).to(rdt)
            tau = 1j * DT  # real time: the step is (0, dt)

            def H(u):
                lap = torch.fft.ifftn(torch.fft.fftn(u) * (-K2))  # ifftn carries the 1/N^3
                dens = u.real * u.real + u.imag * u.imag
                return -0.5 * lap + (C3 * dens + C4 * dens * torch.sqrt(dens)) * u

            def rk4(psi):
                k1 = H(psi)
                k2_ = H(psi - (tau * 0.5) * k1)
                k3 = H(psi - (tau * 0.5) * k2_)
                k4 = H(psi - tau * k3)
                return psi - ((1.0 / 6.0) * tau) * (((k1 + 2 * k2_) + 2 * k3) + k4)

            one = rk4(x0)
            state = {"psi": x0}

            def run():
                state["psi"] = rk4(state["psi"])

            for _ in range(warmup):
                run()
            ms_step = timed(run, steps)
            fft_ms = timed(lambda: torch.fft.ifftn(torch.fft.fftn(x0)), steps)
            one_host = one.cpu().numpy()
            del state, one
        # the product on the same stream: a plan, the forward + inverse pair, one RK4 step
        plan = _abi.Plan(shape, left, right, precision=prec, device=dev)
        plan.set_stream(stream.cuda_stream)
        src, dst = plan.field(psi0), plan.field()

        def pair():
            plan.fft(src, dst, _abi.GP5_FORWARD)
            plan.fft(dst, dst, _abi.GP5_BACKWARD)

        for _ in range(warmup):
            pair()
        ours_fft_ms = timed(pair, steps)
        func = _abi.Functional(plan, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
        st = _abi.Stepper(func, DT, _abi.GP5_STEP_RK4, imaginary=False)
        f = plan.field(psi0)
        st.advance(f, 1)
        mine = f.download()[..., 0].transpose(2, 1, 0)
        diff = float(np.max(np.abs(mine - one_host)) / np.max(np.abs(one_host)))
        out[key] = {"rk4_ms_per_step": ms_step, "value": n ** 3 / (ms_step / 1e3), "unit": "site-updates/s",
                    "fft3d_pair_ms": {"cufft": fft_ms, "gp5cu_fft": ours_fft_ms},
                    "one_step_rel_diff_vs_product": diff}
        del f, st, func, src, dst, plan, x0, K2
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return out


def roofline(r, dtype: str = "c128"):
    """Dominant kernel (largest share of a step) with its algorithmic bytes per launch."""
    prof = r["profile"]
    F = r["field_bytes"]
    bytes_per = []
    kinds = [k for k, _ in prof]
    if len(prof) == 20:
        for s in range(4):
            bytes_per += [STAGE_XFWD[s] * F, 2 * F, 2 * F, 2 * F, STAGE_XINV[s] * F]
    elif kinds.count(3) == 4 and kinds[-1] == 3:
        # merged path: per stage, the y/z passes (on `slabs` x-slabs) then the boundary.  With
        # one slab each y/z launch reads and writes the field in HBM; with several, a slab
        # stays in L2 from its y forward pass to its y inverse pass: y forward reads it from
        # HBM, y inverse writes it back, the z pass runs in L2.
        slabs = kinds.count(10) // 4
        stage = 0
        for k in kinds:
            if k == 3:
                bytes_per.append(MERGED_BOUNDARY[stage] * F)
                stage += 1
            elif slabs == 1:
                bytes_per.append(2 * F)
            else:
                bytes_per.append({10: F / slabs, 22: 0.0, 11: F / slabs}[k])
    elif kinds.count(2) in (1, 4) and kinds[-1] == 2 and 3 not in kinds:
        # per-axis kinetic scheme: per stage the y and z derivative passes (on `slabs` x-slabs)
        # then the boundary.  One slab: y reads u and writes T (2F), z reads u and T and writes
        # T (3F); several: a slab's u and T stay in L2 between its y and z passes, so the y pass
        # reads u from HBM and the z pass writes T back.
        slabs = kinds.count(12) // kinds.count(2)
        stage = 0
        bounds = AXES_BOUNDARY if kinds.count(2) == 4 else [4]
        for k in kinds:
            if k == 2:
                bytes_per.append(bounds[stage] * F)
                stage += 1
            elif slabs == 1:
                bytes_per.append({12: 2 * F, 22: 3 * F}[k])
            else:
                bytes_per.append(F / slabs)
    else:
        return None
    tot = {}
    for (kind, ms), b in zip(prof, bytes_per):
        t = tot.setdefault(kind, [0.0, 0.0, 0])
        t[0] += ms
        t[1] += b
        t[2] += 1
    step_ms = sum(ms for _, ms in prof)
    kind, (ms, b, n) = max(tot.items(), key=lambda kv: kv[1][0])
    peak, src = measured_peaks()
    achieved = b / (ms / 1e3) / 1e9
    name = KIND_NAMES.get(kind, str(kind))
    traffic = ncu_traffic(name, dtype)
    step_bytes = sum(bytes_per)
    return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "peak_source": src, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "algorithmic_bytes_per_launch": b / n, "launches_per_step": n,
            "share_of_step": round(ms / step_ms, 4),
            "step": {"algorithmic_bytes": step_bytes, "bytes_per_site": step_bytes / N_GRID ** 3,
                     "achieved": round(step_bytes / (step_ms / 1e3) / 1e9, 1),
                     "frac": round(step_bytes / (step_ms / 1e3) / 1e9 / peak, 4)},
            "per_kind_ms": {KIND_NAMES.get(k, str(k)): round(v[0], 4) for k, v in tot.items()}}


# ---- precision report (complex64 bulk against complex128) ----------------------------------
def precision_report(dev: int, steps: int = 5000, every: int = 500, tol: float = 1e-8):
    """Ground state at c3 = -3 (imaginary-time RK4 to the residual tol, complex128), then the
    quench c3 -> -3.3 in real time for `steps` RK4 steps of dt = 5e-5 in complex128 and in
    complex64 from the same state (three complex64 forms: as created, with the stochastically
    rounded state update; compensated; rounded to nearest); every `every` steps the norm and
    the energy (FP64 reductions) and each complex64 form's energy error against complex128."""
    import numpy as np
    import torch

    from gp5_b200 import _abi

    torch.cuda.set_device(dev)
    shape, left, right = workload_geometry()
    dx = (right[0] - left[0]) / N_GRID
    p64 = _abi.Plan(shape, left, right, precision=_abi.GP5_C128, device=dev)
    fgs = _abi.Functional(p64, _abi.GP5_FUNC_LHY, c3=-3.0, c4=C4)
    sgs = _abi.Stepper(fgs, 0.15 * dx * dx, _abi.GP5_STEP_RK4, imaginary=True)
    sgs.set_renormalization([N_ATOMS])
    f = p64.field(initial_state())
    t0 = time.perf_counter()
    gs_steps = 0
    ob = fgs.observables(f)
    while ob["residual"] > tol and gs_steps < 100000:
        sgs.advance(f, 500)
        gs_steps += 500
        ob = fgs.observables(f)
    gs = {"steps": gs_steps, "residual": ob["residual"], "energy": ob["energy"], "mu": ob["mu"],
          "seconds": round(time.perf_counter() - t0, 1)}
    psi0 = f.download()
    del f, sgs, fgs
    rows = {}
    f_eval = _abi.Functional(p64, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)  # complex128 evaluation
    e_field = p64.field()
    p32 = None
    ms_adv = {}
    for prec, name, form in ((_abi.GP5_C128, "c128", ""), (_abi.GP5_C64, "c64", ""),
                             (_abi.GP5_C64, "c64c", "comp"), (_abi.GP5_C64, "c64rn", "rn")):
        if prec == _abi.GP5_C128:
            p = p64
        else:
            p32 = p32 or _abi.Plan(shape, left, right, precision=prec, device=dev)
            p = p32
        fq = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
        sq = _abi.Stepper(fq, DT, _abi.GP5_STEP_RK4, imaginary=False)
        if form == "comp":
            sq.set_compensation(True)
        elif form == "rn":
            sq.set_stochastic_rounding(False)
        g = p.field(psi0)
        out = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tms = []
        for k in range(0, steps + 1, every):
            if k:
                torch.cuda.synchronize()
                e0.record()
                sq.advance(g, every)
                e1.record()
                torch.cuda.synchronize()
                tms.append(e0.elapsed_time(e1) / every)
            o = fq.observables(g)
            e128 = o["energy"]
            if prec == _abi.GP5_C64:
                # the complex64 state evaluated by the complex128 functional
                e_field.upload(np.asarray(g.download(), dtype=np.complex128))
                e128 = f_eval.observables(e_field)["energy"]
            out.append((k, o["norm"], o["energy"], e128))
        rows[name] = out
        ms_adv[name] = sorted(tms)[len(tms) // 2] if tms else None  # median ms per step (graph, warm)
        del g, sq, fq
    table = []
    n0 = rows["c128"][0][1]
    for (k, n64, e64, _), (_, n32, e32, e32s), (_, nc, ec, ecs), (_, nr, er, ers) in zip(
            rows["c128"], rows["c64"], rows["c64c"], rows["c64rn"]):
        table.append({"step": k, "norm_c128": n64, "norm_c64": n32, "norm_c64c": nc, "norm_c64rn": nr,
                      "energy_c128": e64, "energy_c64": e32, "energy_c64c": ec, "energy_c64rn": er,
                      "energy_c64_state_in_c128": e32s, "energy_c64c_state_in_c128": ecs,
                      "energy_c64rn_state_in_c128": ers,
                      "norm_drift_c128": (n64 - n0) / n0, "norm_drift_c64": (n32 - n0) / n0,
                      "norm_drift_c64c": (nc - n0) / n0, "norm_drift_c64rn": (nr - n0) / n0,
                      "energy_rel_err_c64": abs(e32 - e64) / abs(e64),
                      "energy_rel_err_c64_state": abs(e32s - e64) / abs(e64),
                      "energy_rel_err_c64c": abs(ec - e64) / abs(e64),
                      "energy_rel_err_c64c_state": abs(ecs - e64) / abs(e64),
                      "energy_rel_err_c64rn": abs(er - e64) / abs(e64),
                      "energy_rel_err_c64rn_state": abs(ers - e64) / abs(e64)})
    return {"ground_state": gs, "checkpoints": table, "ms_per_step_median": ms_adv,
            "max_energy_rel_err_c64c": max(r["energy_rel_err_c64c"] for r in table),
            "max_norm_drift_c64c": max(abs(r["norm_drift_c64c"]) for r in table),
            "max_energy_rel_err_c64": max(r["energy_rel_err_c64"] for r in table),
            "max_energy_rel_err_c64_state": max(r["energy_rel_err_c64_state"] for r in table),
            "max_energy_rel_err_c64c_state": max(r["energy_rel_err_c64c_state"] for r in table),
            "max_energy_rel_err_c64rn": max(r["energy_rel_err_c64rn"] for r in table),
            "max_energy_rel_err_c64rn_state": max(r["energy_rel_err_c64rn_state"] for r in table),
            "max_norm_drift_c64rn": max(abs(r["norm_drift_c64rn"]) for r in table),
            "max_norm_drift_c128": max(abs(r["norm_drift_c128"]) for r in table),
            "max_norm_drift_c64": max(abs(r["norm_drift_c64"]) for r in table),
            "workload": "N=5000 LHY droplet, 256^3, L=4 N^(1/3); ground state at c3=-3 (residual 1e-8), "
                        "quench to c3=-3.3, real-time RK4 dt=5e-5"}


def precision_check(dev: int, steps: int = 500, every: int = 100):
    """complex64 (as created: stochastic state rounding; compensated; rounded to nearest) against
    complex128 on the bench workload itself: the
    same initial state, `steps` real-time RK4 steps of the quenched droplet in each precision;
    every `every` steps the norm and the energy (FP64 reductions, complex64 state evaluated by
    the complex128 functional) against the complex128 run.  Returns the maxima."""
    import numpy as np

    from gp5_b200 import _abi

    shape, left, right = workload_geometry()
    psi0 = initial_state()
    p64 = _abi.Plan(shape, left, right, precision=_abi.GP5_C128, device=dev)
    p32 = _abi.Plan(shape, left, right, precision=_abi.GP5_C64, device=dev)
    f_eval = _abi.Functional(p64, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
    e_field = p64.field()
    rows = {}
    for name, p, form in (("c128", p64, ""), ("c64", p32, ""), ("c64c", p32, "comp"), ("c64rn", p32, "rn")):
        fq = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
        sq = _abi.Stepper(fq, DT, _abi.GP5_STEP_RK4, imaginary=False)
        if form == "comp":
            sq.set_compensation(True)
        elif form == "rn":
            sq.set_stochastic_rounding(False)
        g = p.field(psi0)
        out = []
        for k in range(0, steps + 1, every):
            if k:
                sq.advance(g, every)
            if p is p64:
                o = f_eval.observables(g)
            else:
                e_field.upload(np.asarray(g.download(), dtype=np.complex128))
                o = f_eval.observables(e_field)
            out.append((o["norm"], o["energy"]))
        rows[name] = out
        del g, sq, fq
    ref = rows["c128"]
    n0 = ref[0][0]
    res = {"steps": steps, "every": every,
           "max_norm_drift_c128": max(abs(n - n0) / n0 for n, _ in ref)}
    for name in ("c64", "c64c", "c64rn"):
        res["max_energy_rel_err_" + name] = max(abs(e - er) / abs(er) for (_, e), (_, er) in zip(rows[name], ref))
        res["max_norm_drift_" + name] = max(abs(n - n0) / n0 for n, _ in rows[name])
    res["workload"] = ("bench workload (Gaussian start, c3=-3.3), real-time RK4 dt=5e-5 in each precision "
                       "from the same state; complex64 states evaluated in complex128")
    return res


# ---- batched droplet ground states (config: 64 seeded solves; bench leg: a seeded sample) ----
def batch_solves(count: int, seed: int = 2025, rank: int = 0):
    """N log-uniform in [20, 2000], c3 ~ U[-3.2, -2.8], c4 = 2.5, no trap, L = 4 N^(1/3); grid:
    the smallest of 32^3/64^3/128^3 with L/n <= 0.25, else 128^3 (N > 512 cannot meet the
    spacing on these grids); dt = 0.15 dx^2 (RK4 is stable on the cube-corner modes
    K^2 = 3 (pi/dx)^2 up to dt = 0.188 dx^2)."""
    import numpy as np

    # each rank draws its own shard of droplets (independent solves: no data-path collective)
    rng = np.random.default_rng([seed, rank])
    out = []
    for _ in range(count):
        N = float(np.exp(rng.uniform(math.log(20.0), math.log(2000.0))))
        c3 = float(rng.uniform(-3.2, -2.8))
        L = 4.0 * N ** (1.0 / 3.0)
        n = next((m for m in (32, 64, 128) if L / m <= 0.25), 128)
        dx = L / n
        out.append(dict(n=n, L=L, N=N, c3=c3, c4=2.5, omega=0.0, dt=0.15 * dx * dx))
    return out


def droplet_state(sd, seed):
    import numpy as np

    n, L, N = sd["n"], sd["L"], sd["N"]
    x = -L / 2 + L / n * (np.arange(n) + 0.5)
    sig = 0.5 * N ** (1.0 / 3.0)
    g = np.exp(-x * x / (2 * sig * sig))
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.complex128)
    psi *= np.exp(1j * 1e-3 * np.random.default_rng(seed).uniform(-1, 1, psi.shape))
    psi *= math.sqrt(N / (float(np.sum(np.abs(psi) ** 2)) * (L / n) ** 3))
    return np.asfortranarray(psi)


def run_batch(count: int, dev: int, tol: float = 1e-8, rank: int = 0, world: int = 1, precision: str = "c128",
              method: str = "rk4"):
    import torch

    from gp5_b200 import _abi

    solves = batch_solves(count, rank=rank)
    prec = _abi.GP5_C128 if precision == "c128" else _abi.GP5_C64
    b = _abi.Batch(solves, precision=prec, device=dev)
    check_every = 500
    if method == "precond":
        b.set_method(_abi.GP5_BATCH_PRECOND, 0.5)
        check_every = 5
    for k, sd in enumerate(solves):
        b.set_state(k, droplet_state(sd, 3000 + 1000 * rank + k))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    res = b.solve(tol=tol, check_every=check_every, max_steps=400000)
    wall = max_over_ranks(time.perf_counter() - t0, world)
    conv = int(sum_over_ranks(sum(r["converged"] for r in res), world))
    site_steps = sum_over_ranks(sum(r["steps"] * sd["n"] ** 3 for r, sd in zip(res, solves)), world)
    launches = int(sum_over_ranks(b.launches, world))
    grids = {}
    for sd in solves:
        grids[str(sd["n"])] = grids.get(str(sd["n"]), 0) + 1
    out = {"value": conv / wall, "unit": "ground states/s", "solves": count * world, "converged": conv,
           "tol": tol, "seconds": wall, "dtype": precision, "grids_rank0": grids,
           "steps_rank0": {"min": min(r["steps"] for r in res), "max": max(r["steps"] for r in res),
                           "mean": sum(r["steps"] for r in res) / count},
           "site_updates_per_s": site_steps / wall, "gpu_launches": launches,
           "energies_rank0": [r["energy"] for r in res],
           "workload": "seeded LHY droplets (one shard of " + str(count) + " per rank): N log-uniform "
                       "[20,2000], c3 U[-3.2,-2.8], c4 2.5, Gaussian start (width 0.5 N^(1/3), phase "
                       "noise 1e-3), imaginary-time RK4 renormalised every step, dt 0.15 dx^2, residual "
                       "checked every 500 steps"}
    if method == "precond":
        out["workload"] = out["workload"].replace(
            "imaginary-time RK4 renormalised every step, dt 0.15 dx^2, residual checked every 500 steps",
            "preconditioned gradient iteration (gp5cu_batch_set_method GP5_BATCH_PRECOND, theta 0.5), "
            "residual checked every 5 iterations; steps count iterations")
    if precision == "c64":
        out["steps_c64_rank0_mean"] = sum(r["steps_c64"] for r in res) / count
        out["method"] = ("complex64 state and transforms (FP64 reductions) until the residual reaches 1e-5 "
                         "or stops falling, then complex128 to the tolerance")
    out["_steps"] = [r["steps"] for r in res]
    out["_grids"] = [sd["n"] for sd in solves]
    return out


def cpu_ground_state_baseline(gs: dict, seconds_per_grid: float = 4.0):
    """Ground states/s of the oracle (the reference's arithmetic: renormalised imaginary-time
    RK4, all host threads) on the same seeded droplets, extrapolated: for every grid size of the
    batch, the time of one oracle RK4 step is measured on a bounded sample of steps of a
    droplet of that grid, and each solve is charged the steps the GPU solver needed for it
    (the same algorithm in the same arithmetic takes the same steps)."""
    import numpy as np

    from oracle import gp_oracle as o

    o.set_elementwise_threads(o._WORKERS)
    per_step = {}
    sample = []
    for n in sorted(set(gs["_grids"])):
        sd = next(s for s in batch_solves(len(gs["_grids"])) if s["n"] == n)
        geo = o.Geometry((n,) * 3, (-sd["L"] / 2,) * 3, (sd["L"] / 2,) * 3)
        psi = np.asfortranarray(droplet_state(sd, 1)[..., None])
        st = o.Stepper(o.Functional("lhy", c3=sd["c3"], c4=sd["c4"]), geo, sd["dt"], "RK4", imaginary=True,
                       normalizations=[sd["N"]])
        psi = st.advance(psi, 1)  # warm
        k, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < seconds_per_grid or k < 2:
            psi = st.advance(psi, 1)
            k += 1
        per_step[n] = (time.perf_counter() - t0) / k
        sample.append(f"{k} RK4 steps at {n}^3")
    total = sum(steps * per_step[n] for steps, n in zip(gs["_steps"], gs["_grids"]))
    return {"value": len(gs["_steps"]) / total, "unit": "ground states/s", "cores": o._WORKERS, "kind": "port",
            "seconds_per_step": {str(n): t for n, t in per_step.items()},
            "sample": "; ".join(sample) + "; extrapolated to the GPU solver's step count of every solve "
                      f"({sum(gs['_steps'])} steps in total, {total:.0f} s on the host)"}


def cpu_precond_baseline(gp: dict, iters: int = 10):
    """Ground states/s of the oracle's preconditioned iteration (oracle.gp_oracle.
    precond_ground_state: the same method in FP64 numpy, all host threads) on the same droplets,
    extrapolated like cpu_ground_state_baseline: the time of `iters` iterations (with a residual
    check every 5, as on the GPU) per grid size, charged with the GPU's iteration count of every
    solve."""
    import numpy as np

    from oracle import gp_oracle as o

    o.set_elementwise_threads(o._WORKERS)
    per_iter = {}
    for n in sorted(set(gp["_grids"])):
        sd = next(s for s in batch_solves(len(gp["_grids"])) if s["n"] == n)
        geo = o.Geometry((n,) * 3, (-sd["L"] / 2,) * 3, (sd["L"] / 2,) * 3)
        psi = np.asfortranarray(droplet_state(sd, 1)[..., None])
        func = o.Functional("lhy", c3=sd["c3"], c4=sd["c4"])
        t0 = time.perf_counter()
        o.precond_ground_state(func, geo, psi, sd["N"], tol=0.0, check_every=5, max_iter=iters)
        per_iter[n] = (time.perf_counter() - t0) / iters
    total = sum(k * per_iter[n] for k, n in zip(gp["_steps"], gp["_grids"]))
    return {"value": len(gp["_steps"]) / total, "unit": "ground states/s", "cores": o._WORKERS, "kind": "port",
            "seconds_per_iteration": {str(n): t for n, t in per_iter.items()},
            "sample": f"{iters} iterations per grid size; extrapolated to the GPU solver's iteration count of "
                      f"every solve ({sum(gp['_steps'])} in total, {total:.0f} s on the host)"}


def cpu_reference_timing(max_seconds: float, max_steps: int, warmup: int = 1):
    """RK4 steps of the oracle (the reference's arithmetic) on the host, all threads: `warmup`
    untimed steps, then up to `max_steps` timed steps or `max_seconds`, whichever ends first."""
    from oracle import gp_oracle as o

    shape, left, right = workload_geometry()
    geo = o.Geometry(shape, left, right)
    psi = initial_state()
    # every host thread: the transforms through scipy.fft's workers, the element-wise work over
    # z-slabs (the reference spreads both over its MPI ranks)
    o.set_elementwise_threads(o._WORKERS)
    st = o.Stepper(o.Functional("lhy", c3=C3, c4=C4), geo, DT, "RK4", imaginary=False)
    if warmup > 0:
        psi = st.advance(psi, warmup)
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        psi = st.advance(psi, 1)
        n += 1
        if time.perf_counter() - t0 > max_seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": N_GRID ** 3 * n / dt, "unit": "site-updates/s", "cores": o._WORKERS, "kind": "port",
            "steps": n, "seconds": dt, "warmup": warmup,
            "sample": f"{n} RK4 step(s) of the 256^3 complex128 workload; scipy.fft with "
                      f"{o._WORKERS} workers, element-wise numpy over {o._WORKERS} threads"}


def profiling_case(what: str) -> None:
    """Small cases for ncu captures of single kernels (fields of 134-268 MB, above L2; about
    1 GB on the device): step64 / step128 advance the bench workload two RK4 steps in
    complex64 / complex128, obs128 evaluates the observables and the norm twice (the
    point-wise reductions), cluster labels the droplets of the start state twice."""
    import numpy as np

    from gp5_b200 import _abi

    shape, left, right = workload_geometry()
    psi0 = initial_state()
    if what in ("step64", "step128"):
        prec = _abi.GP5_C64 if what == "step64" else _abi.GP5_C128
        p = _abi.Plan(shape, left, right, precision=prec)
        f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
        st = _abi.Stepper(f, DT, _abi.GP5_STEP_RK4, imaginary=False)
        a = p.field(psi0)
        st.advance(a, 2)
        print("radix", p.radix(), "tiles", p.tiles(), "launches per step", st.launches_per_step)
    elif what == "obs128":
        p = _abi.Plan(shape, left, right)
        f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=C3, c4=C4)
        a = p.field(psi0)
        for _ in range(2):
            print(f.observables(a), p.norm(a))
    else:
        p = _abi.Plan(shape, left, right)
        a = p.field(psi0)
        cut = 0.5 * float(np.max(np.abs(psi0)) ** 2)
        for _ in range(2):
            print("clusters", p.decompose(a, cut)[1])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision-check", action="store_true",
                    help="skip the 500-step complex64-vs-complex128 energy check (profiling runs)")
    ap.add_argument("--min-seconds", type=float, default=2.0,
                    help="repeat the timed K steps until this much timed work has passed (clock sampling)")
    ap.add_argument("--precision-report", metavar="JSON",
                    help="also run the complex64-vs-complex128 quench report and write it here")
    ap.add_argument("--batch", type=int, default=64,
                    help="solves of the ground-state leg, in complex128 and in complex64 (0: skip)")
    ap.add_argument("--no-comparator", action="store_true",
                    help="skip the cuFFT comparator (torch.fft RK4 step and transform pair)")
    ap.add_argument("--case", choices=["step64", "step128", "obs128", "cluster"],
                    help="run one small profiling case of the workload and exit (no JSON line)")
    args = ap.parse_args()
    if args.case:
        profiling_case(args.case)
        return
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": "LHY droplet quench, real-time RK4, 256^3, N=5000, L=4 N^(1/3), c3=-3.3, c4=2.5, "
                          "dt=5e-5", "grid": [N_GRID] * 3, "precision_leg": ["complex128", "complex64"],
              "l2": "inputs larger than L2 (each field 256 MiB)", "parallelism": f"replicas x{world}"}
    metric = "RK4 site-updates/s at 256^3 (FP64; FP32 in 'fp32')"

    if args.impl == "reference":
        if rank != 0:
            return
        # a bounded sample: at most ~150 s of timed CPU steps (one step of the oracle at 256^3
        # takes about a second on 16 host threads)
        r = cpu_reference_timing(max_seconds=150.0, max_steps=args.steps, warmup=args.warmup)
        line = {"impl": "reference", "metric": metric, "value": r["value"], "unit": "site-updates/s",
                "n_gpus": args.gpus, "steps": r["steps"], "warmup": r["warmup"],
                "ms_per_step": r["seconds"] / r["steps"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                "data": "synthetic", "config": config,
                "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": r["value"], "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import datetime

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device(f"cuda:{local_rank}"))
    results, launches = run_ours(args, rank, world, local_rank)
    gs = None
    if args.batch > 0:
        # the configuration's solves are shared out over the ranks (each draws its own seeded
        # shard), so a run on N GPUs solves about the same number of droplets as one on 1 GPU
        per_rank = max(1, args.batch // world)
        gs = run_batch(per_rank, local_rank, rank=rank, world=world, precision="c128")
        gs["c64"] = run_batch(per_rank, local_rank, rank=rank, world=world, precision="c64")
        # the same droplets by the preconditioned iteration (a different method to the same
        # ground states: not the configuration's imaginary-time workload, reported beside it)
        gs["preconditioned"] = run_batch(per_rank, local_rank, rank=rank, world=world, precision="c128",
                                         method="precond")
    comparator = None
    if world == 1 and not args.no_comparator:
        comparator = cufft_comparator(local_rank)
    prep = None
    if args.precision_report and world == 1:
        prep = precision_report(local_rank)
        with open(args.precision_report, "w") as fh:
            json.dump(prep, fh, indent=1)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    r64, r32, r32c, r32n = results[0], results[1], results[2], results[3]
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        c = cpu_reference_timing(max_seconds=20.0, max_steps=4, warmup=0)
        cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if gs is not None:
        if world == 1 and not args.no_cpu_baseline:
            gs["cpu_baseline"] = cpu_ground_state_baseline(gs)
            gs["preconditioned"]["cpu_baseline"] = cpu_precond_baseline(gs["preconditioned"])
        e128 = gs.pop("energies_rank0")
        e64 = gs["c64"].pop("energies_rank0")
        gs["c64"]["max_energy_rel_diff_vs_c128"] = max(abs(a - b) / abs(b) for a, b in zip(e64, e128))
        ep = gs["preconditioned"].pop("energies_rank0")
        gs["preconditioned"]["max_energy_rel_diff_vs_rk4"] = max(abs(a - b) / abs(b) for a, b in zip(ep, e128))
        gs["preconditioned"]["speedup_vs_rk4"] = gs["preconditioned"]["value"] / gs["value"]
        for d in (gs, gs["c64"], gs["preconditioned"]):
            d.pop("_steps")
            d.pop("_grids")
    energy = ({k: prep[k] for k in ("max_energy_rel_err_c64", "max_energy_rel_err_c64_state", "max_energy_rel_err_c64c",
                                    "max_energy_rel_err_c64c_state", "max_energy_rel_err_c64rn",
                                    "max_energy_rel_err_c64rn_state", "max_norm_drift_c64c", "max_norm_drift_c64rn",
                                    "ms_per_step_median", "max_norm_drift_c64", "max_norm_drift_c128")} if prep else
              (None if args.no_precision_check else precision_check(local_rank)))
    line = {"metric": metric, "value": r64["value"], "unit": "site-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r64["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic", "config": config,
            "fp32": {"value": r32["value"], "ms_per_step": r32["ms_per_step"], "dtype": "c64",
                     "speedup_vs_fp64": r32["value"] / r64["value"], "clocks": r32["clocks"],
                     "roofline": roofline(dict(r32, field_bytes=r64["field_bytes"] // 2), "c64"),
                     "energy_error": energy,
                     "state_rounding": "stochastic (the complex64 default, gp5cu_stepper_set_stochastic_rounding)",
                     "compensated": {"value": r32c["value"], "ms_per_step": r32c["ms_per_step"],
                                     "speedup_vs_fp64": r32c["value"] / r64["value"], "clocks": r32c["clocks"],
                                     "note": "gp5cu_stepper_set_compensation: BF16 correction field, "
                                             "two-sum state update"},
                     "round_to_nearest": {"value": r32n["value"], "ms_per_step": r32n["ms_per_step"],
                                          "speedup_vs_fp64": r32n["value"] / r64["value"],
                                          "clocks": r32n["clocks"],
                                          "note": "gp5cu_stepper_set_stochastic_rounding(0)"}},
            "e2e": r64["e2e"], "roofline": roofline(r64, "c128"), "cpu_baseline": cpu,
            "clocks": r64["clocks"], "gpu_launches": launches,
            "autotune": {"passes": ["y_fwd", "y_inv", "z_fwd", "z_inv", "z_fwd_kinetic_inv"],
                         "threads_per_cta": {"c128": r64["tiles"], "c64": r32["tiles"]}}, "ground_states": gs,
            "launches_per_step": r64["launches_per_step"]}
    if comparator is not None:
        for key, r in (("c128", r64), ("c64", r32)):
            comparator[key]["product_over_comparator"] = r["value"] / comparator[key]["value"]
        line["cufft_comparator"] = comparator
    print(json.dumps(line))


if __name__ == "__main__":
    main()
