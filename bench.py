#!/usr/bin/env python
"""Benchmark: adjoint-state FWI gradient seconds per shot on the 2D acoustic
workload (201 x 401 grid, dx 10 m, 20-cell CFS-PML, 8th order, dt 1 ms, 2000
steps, 32 shots with offset-truncated receiver spreads, L2 waveform misfit,
every-50-step checkpoints).

One step = one batched gradient over the 32 shots of a GPU (forward with a
checkpoint every 50 steps, the last segment's stencil terms stored by the
forward; residual + FP64 misfit; reverse sweep recomputing each earlier segment
from its checkpoint, then the exact adjoint through it; FP64 chain rule). With
N GPUs the shot set has 32 N shots, sharded over the ranks by trace count; the
gradient and the per-shot misfits are summed over ranks in FP64 with one NCCL
all-reduce each per step.

Prints one JSON line (rank 0). ``--impl reference`` times the reference's own
CPU gradient algorithm (restated loops, OpenMP on all host threads) instead:
one step = the full 2000-step gradient of one shot.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NSHOTS = 32


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="owl", choices=["owl", "reference"])
    p.add_argument("--no-plain", action="store_true", help="skip the per-shot plain-path measurement")
    p.add_argument("--no-check", action="store_true", help="skip the FP64-oracle gradient check")
    p.add_argument("--nshots", type=int, default=NSHOTS, help="shots per GPU (32 for the benchmark)")
    p.add_argument("--profile", action="store_true",
                   help="profiling target: one gradient step of --nshots shots, nothing else, no JSON line")
    p.add_argument("--tile-z", type=int, default=0,
                   help="--profile / --profile-el: tile code of the kernels (--profile 0: autotuned, which adds "
                        "the tuning launches; --profile-el 0: 8)")
    p.add_argument("--spt", type=int, default=0, help="--profile: shots per CTA with --tile-z")
    p.add_argument("--no-3d", action="store_true", help="skip the 3D acoustic forward roofline block")
    p.add_argument("--no-misfits", action="store_true", help="skip the data-domain misfit block")
    p.add_argument("--rows", type=int, default=1, help="rows per thread of the --profile3d forward kernels")
    p.add_argument("--profile3d", type=int, default=0, metavar="N",
                   help="profiling target: 12-step 3D acoustic forward of an N^3 model, no JSON line")
    p.add_argument("--profile3d-grad", type=int, default=0, metavar="N",
                   help="profiling target: one 3D acoustic gradient of an N^3 model, 1 shot, 60 steps, no JSON line")
    p.add_argument("--no-elastic", action="store_true", help="skip the 2D elastic VTI block")
    p.add_argument("--el3-grad-shots", type=int, default=16,
                   help="shots of the 3D elastic gradient at the workload's size (0: none)")
    p.add_argument("--profile-el", type=int, default=0, metavar="S",
                   help="profiling target: one 2D elastic VTI gradient of S shots, 60 steps, no JSON line")
    p.add_argument("--ring", action="store_true", help="--profile-el3 with the ring forward kernels")
    p.add_argument("--profile-el3-fwd", type=int, default=0, metavar="N",
                   help="profiling target: a 10-step 3D elastic ORT forward of 1 shot on an N^3 model")
    p.add_argument("--profile-el3", type=int, default=0, metavar="N",
                   help="profiling target: one 3D elastic ORT gradient of 1 shot on an N^3 model, 40 steps")
    return p.parse_args()


def profile_3d(n, rows=1):
    """Small 3D forward for kernel captures: N^3 layered model, one shot, 12 steps,
    forward tiles fixed at `rows` rows per thread (no autotuning launches)."""
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.geometry import Receiver, Shot, Source
    from owl_b200.solver import RunOpts, SSGSolver

    vp, rho = configs.acoustic_3d_model(n, 10.0)
    c = n // 2 * 10.0
    shots = [Shot(1, [Source(x=c, y=c, z=20.0, f0=12.0)], [Receiver(x=20.0 * i, y=c, z=20.0) for i in range(n // 2)])]
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, n, n, 10.0, 10.0, 1e-3, 12, pml=20, f0_max=12.0, ny=n, dy=10.0)
    s.set_model(vp, rho)
    s.forward(s.prepare(shots), RunOpts(shots_per_cta=1, tile_z=rows, use_graph=-1))
    print(f"profile3d: {s.last_info.elapsed_ms:.2f} ms, {s.last_info.gpu_launches} launches")
    s.close()


def profile_3d_grad(n):
    """Small 3D acoustic gradient for kernel captures: N^3 layered model, one
    shot, 60 steps, checkpoints every 20 steps, the ring kernels of both passes
    (tile_z 1: no autotuning launches)."""
    import numpy as np
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.solver import RunOpts, SSGSolver

    d, vp, rho, shots = configs.config3(n, nt=60)
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, ny=d.ny, dy=d.dy)
    s.set_model(vp, rho)
    ps = s.prepare(shots)
    obs = np.zeros(s.seis_size(ps), dtype=np.float32)
    s.gradient(ps, obs, opts=RunOpts(checkpoint_interval=20, shots_per_cta=1, tile_z=1, use_graph=-1))
    print(f"profile3d-grad: {s.last_info.elapsed_ms:.2f} ms, {s.last_info.gpu_launches} launches")
    s.close()


def forward_3d_block(peak, peak_kind):
    """3D acoustic forward of the 400^3 workload (440^3 padded cells, 1500 steps,
    one shot, 40,000 receivers): Gcell-updates/s of the whole forward and the
    HBM roofline of its two stencil kernels (standalone launches, CUDA events)."""
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.solver import RunOpts, SSGSolver

    d, vp, rho, shots = configs.config3(400, nt=1500)
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, ny=d.ny, dy=d.dy)
    s.set_model(vp, rho)
    ps = s.prepare(shots)
    s.forward(ps, RunOpts())
    ms = []
    for _ in range(2):
        s.forward(ps, RunOpts())
        ms.append(s.last_info.elapsed_ms)
    cells = float(d.nx + 2 * d.pml) ** 3
    out = {"workload": "3D acoustic forward, 400^3 model (440^3 padded), dt 1 ms, 1500 steps, 1 shot, "
                       "40,000 receivers", "ms_per_forward": sum(ms) / len(ms),
           "gcells_per_s": cells * d.nt / (sum(ms) / len(ms) / 1e3) / 1e9,
           "tile_rows_per_thread": s.last_info.tile_z, "kernels": {}}
    for kid, name in ((L.OWL_K_FWD_P, "k_ac3d_fwd_p"), (L.OWL_K_FWD_V, "k_ac3d_fwd_v")):
        kms, b = s.kernel_time(kid, 20)
        ach = b / (kms / 1e3) / 1e9
        out["kernels"][name + " (autotuned variant)"] = {
            "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_source": peak_kind,
            "alg_bytes_per_launch": b, "ms_per_launch": kms, "traffic": profile_traffic(name)}
    s.close()
    # each ring variant on its own (2 rows per thread): 16-byte cp.async copies
    # issued by every thread, or one TMA load per tile completing on an mbarrier
    dk, vpk, rhok, shk = configs.config3(400, nt=8)
    sk = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, dk.nx, dk.nz, dk.dx, dk.dz, dk.dt, dk.nt, pml=dk.pml, fdhalf=dk.fdhalf,
                   f0_max=dk.f0_max, ny=dk.ny, dy=dk.dy)
    sk.set_model(vpk, rhok)
    pk = sk.prepare(shk)
    for tz, tag in ((2, "<4,2> cp.async ring"), (12, "_tma<4,2> TMA ring")):
        sk.forward(pk, RunOpts(tile_z=tz))
        for kid, name in ((L.OWL_K_FWD_P, "k_ac3d_fwd_p"), (L.OWL_K_FWD_V, "k_ac3d_fwd_v")):
            kms, b = sk.kernel_time(kid, 20)
            ach = b / (kms / 1e3) / 1e9
            nm = name + tag.split(" ")[0]
            out["kernels"][nm] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                  "peak_source": peak_kind, "alg_bytes_per_launch": b, "ms_per_launch": kms,
                                  "copies": " ".join(tag.split(" ")[1:]), "traffic": profile_traffic(nm.split("<")[0])}
    sk.close()
    # gradient of the same model and shot over all 1500 steps (FP16 checkpoints
    # every 50 steps), observed data from a 3 % faster model
    import numpy as np
    dg, vpg, rhog, shg = configs.config3(400, nt=1500)
    g = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, dg.nx, dg.nz, dg.dx, dg.dz, dg.dt, dg.nt, pml=dg.pml, fdhalf=dg.fdhalf,
                  f0_max=dg.f0_max, ny=dg.ny, dy=dg.dy)
    pg = g.prepare(shg)
    g.set_model((vpg * np.float32(1.03)).astype(np.float32), rhog)
    obs = g.forward(pg, RunOpts())
    g.set_model(vpg, rhog)
    go = RunOpts(checkpoint_precision=L.OWL_CKPT_FP16)
    g.gradient(pg, obs, opts=go)
    _, gr = g.gradient(pg, obs, opts=go)
    out["gradient_workload"] = "the same model and shot, all 1500 steps, FP16 checkpoints every 50 steps"
    out["gradient_s_per_shot"] = g.last_info.elapsed_ms / 1e3
    out["gradient_finite"] = bool(np.all(np.isfinite(np.asarray(gr))))
    # the autotuner's adjoint kernels: z-marching ring (tile 1) or tiled
    ring = g.last_info.tile_z == 1
    out["adjoint_kernels"] = "z-marching ring" if ring else f"tiled, {g.last_info.tile_z} rows"
    for kid, name in ((L.OWL_K_ADJ_P, "k_ac3d_adj_p_ring" if ring else "k_ac3d_adj_p"),
                      (L.OWL_K_ADJ_V, "k_ac3d_adj_v_ring" if ring else "k_ac3d_adj_v")):
        kms, b = g.kernel_time(kid, 10)
        ach = b / (kms / 1e3) / 1e9
        out["kernels"][name] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                "peak_source": peak_kind, "alg_bytes_per_launch": b, "ms_per_launch": kms,
                                "traffic": profile_traffic(name)}
    g.close()
    return out


def elastic_solver(nshots, nt):
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.solver import SSGSolver

    d, f, shots = configs.config4(nshots, nt=nt)
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_2D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  free_surface=True, f0_max=d.f0_max, max_shots=nshots, aniso=d.aniso)
    s.set_model(*f)
    return d, f, s, s.prepare(shots)


def profile_elastic(nshots, tile_z=8):
    """Small elastic gradient for kernel captures: the 2D VTI model, S shots, 60
    steps, tile code tile_z (100 + h: four-cell forward kernels)."""
    import numpy as np
    from owl_b200.solver import RunOpts
    d, f, s, ps = elastic_solver(nshots, 60)
    obs = np.zeros(s.seis_size(ps), dtype=np.float32)
    s.gradient(ps, obs, opts=RunOpts(checkpoint_interval=20, shots_per_cta=1, tile_z=tile_z, use_graph=-1))
    print(f"profile-el: {s.last_info.elapsed_ms:.2f} ms, {s.last_info.gpu_launches} launches")
    s.close()


def profile_elastic3(n, ring=False):
    """Small 3D elastic gradient for kernel captures: the ORT model on n^3, 1 shot, 40 steps;
    forward kernels thread per cell, or the z-marching ring kernels with ring=True."""
    import numpy as np
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.solver import RunOpts, SSGSolver

    d, f, shots = configs.config5(1, nt=40, n=n, nrec=16)
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=1, ny=d.ny, dy=d.dy, aniso=d.aniso)
    s.set_model(*f)
    ps = s.prepare(shots)
    obs = np.zeros(s.seis_size(ps), dtype=np.float32)
    s.gradient(ps, obs, opts=RunOpts(checkpoint_interval=20, shots_per_cta=1, tile_z=1 if ring else 2, use_graph=-1))
    print(f"profile-el3: {s.last_info.elapsed_ms:.2f} ms, {s.last_info.gpu_launches} launches")
    s.close()


def profile_elastic3_forward(n, ring=False):
    """3D elastic forward for DRAM-traffic captures: the ORT model on n^3 (M-PML
    ratios on), 1 shot, 10 steps, no stored stencil terms; ring or per-cell kernels."""
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.solver import RunOpts, SSGSolver

    d, f, shots = configs.config5(1, nt=10, n=n, nrec=16)
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=1, ny=d.ny, dy=d.dy, aniso=d.aniso)
    s.set_model(*f)
    ps = s.prepare(shots)
    s.forward(ps, RunOpts(shots_per_cta=1, tile_z=1 if ring else 2, use_graph=-1))
    print(f"profile-el3-fwd: {s.last_info.elapsed_ms:.2f} ms, {s.last_info.gpu_launches} launches")
    s.close()


def elastic_2d_block(peak, peak_kind, ngrad=16):
    """2D elastic VTI with a free surface (301 x 601, dx 5 m, 4000 steps, Thomsen
    parameters): forward of all 64 shots (Gcell-updates/s) and the HBM roofline
    of its two stencil kernels, gradient of `ngrad` shots (s/shot) and the
    roofline of its two adjoint kernels."""
    import numpy as np
    from owl_b200 import _lib as L
    from owl_b200.solver import RunOpts

    d, f, s, ps = elastic_solver(64, 4000)
    cells = float(d.nx + 2 * d.pml) * (d.nz + d.pml)  # rows from the surface down
    s.forward(ps, RunOpts())
    fwd = []
    for _ in range(2):
        s.forward(ps, RunOpts())
        fwd.append(s.last_info.elapsed_ms)
    fms = sum(fwd) / len(fwd)
    out = {"workload": "2D elastic VTI, 301 x 601 model, dx 5 m, dt 0.5 ms, 4000 steps, PML 20, free surface, "
                       "64 shots (explosion / vertical force), 301 two-component receivers",
           "forward_ms_64_shots": fms, "forward_gcells_per_s": cells * d.nt * 64 / (fms / 1e3) / 1e9,
           "kernels": {}}

    def roof(kid, name, shots):
        kms, b = s.kernel_time(kid, 20)
        ach = b / (kms / 1e3) / 1e9
        out["kernels"][name] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                "peak_source": peak_kind, "alg_bytes_per_launch": b, "ms_per_launch": kms,
                                "shots_per_launch": shots, "traffic": profile_traffic(name)}

    # the forward's kernels on its own 64-shot launch (autotuned: tile codes >=
    # 100 are the four-cell kernels)
    v4 = s.last_info.tile_z_forward >= 100
    out["forward_tile_code"] = s.last_info.tile_z_forward
    roof(L.OWL_K_FWD_P, "k_el2d_fwd_s4" if v4 else "k_el2d_fwd_s", 64)
    roof(L.OWL_K_FWD_V, "k_el2d_fwd_v4" if v4 else "k_el2d_fwd_v", 64)
    from owl_b200 import configs
    sub = s.prepare(configs.config4_shots(64, d.nx, d.dx)[:ngrad])
    obs = np.zeros(s.seis_size(sub), dtype=np.float32)
    opts = RunOpts(checkpoint_precision=L.OWL_CKPT_FP16)
    s.gradient(sub, obs, opts=opts)
    gms = []
    for _ in range(2):
        _, gr = s.gradient(sub, obs, opts=opts)
        gms.append(s.last_info.elapsed_ms)
    out["gradient_finite"] = bool(np.all(np.isfinite(np.asarray(gr))))
    out["gradient_shots"] = ngrad
    out["gradient_s_per_shot"] = sum(gms) / len(gms) / 1e3 / ngrad
    out["gradient_checkpoints"] = "fp16, per-field scale, every 50 steps"
    # the adjoint kernels on the gradient's 16-shot launch
    out["gradient_tile_codes"] = {"forward": s.last_info.tile_z_forward, "adjoint": s.last_info.tile_z}
    roof(L.OWL_K_ADJ_P, "k_el2d_adj_v", ngrad)
    roof(L.OWL_K_ADJ_V, "k_el2d_adj_s", ngrad)
    s.close()
    return out


def elastic_3d_block(peak, peak_kind, nshots=4, nt=500, grad_shots=16):
    """3D elastic orthorhombic (nine Cij) on the 256^3 model (296^3 padded cells):
    forward of `nshots` of the 16 vertical-force shots over `nt` of the 2500
    steps (Gcell-updates/s, HBM roofline of the two forward stencil kernels),
    then the gradient w.r.t. the nine Cij and rho of `grad_shots` shots over all
    2500 steps with FP16 checkpoints, shots per batch and checkpoint interval
    chosen by the memory planner (s/shot, HBM roofline of the two adjoint
    kernels on that gradient's state)."""
    import numpy as np
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.solver import RunOpts, SSGSolver

    d, f, shots = configs.config5(nshots, nt=nt)
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=nshots, ny=d.ny, dy=d.dy, aniso=d.aniso)
    s.set_model(*f)
    ps = s.prepare(shots)
    s.forward(ps, RunOpts())
    s.forward(ps, RunOpts())
    fms = s.last_info.elapsed_ms
    cells = float(d.nx + 2 * d.pml) ** 3
    out = {"workload": f"3D elastic ORT (nine Cij), 256^3 model (296^3 padded), dt 0.8 ms, {nt} of 2500 steps, "
                       f"{nshots} of 16 vertical-force shots, 128 x 128 three-component receivers",
           "forward_ms": fms, "forward_gcells_per_s": cells * nt * nshots / (fms / 1e3) / 1e9, "kernels": {}}
    # the autotuner's forward kernels: z-marching ring (tile_z 1) or thread per
    # cell, timed on one shot per launch (the gradient's batch; the traffic
    # figure is an ncu capture of that launch)
    ring = s.last_info.tile_z == 1
    out["forward_kernels"] = "z-marching ring" if ring else "thread per cell"
    s.forward(s.prepare(shots[:1]), RunOpts(tile_z=1 if ring else 2))
    for kid, name in ((L.OWL_K_FWD_P, "k_el3d_fwd_s_ring" if ring else "k_el3d_fwd_s"),
                      (L.OWL_K_FWD_V, "k_el3d_fwd_v_ring" if ring else "k_el3d_fwd_v")):
        kms, b = s.kernel_time(kid, 10)
        ach = b / (kms / 1e3) / 1e9
        out["kernels"][name] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                "peak_source": peak_kind, "alg_bytes_per_launch": b, "ms_per_launch": kms,
                                "shots_per_launch": 1, "traffic": profile_traffic(name)}
    s.close()
    if grad_shots <= 0:
        return out
    # the gradient at the workload's size: all 2500 steps, FP16 checkpoints
    dg, fg, shg = configs.config5(16, nt=2500)
    shg = shg[:grad_shots]
    g = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, dg.nx, dg.nz, dg.dx, dg.dz, dg.dt, dg.nt, pml=dg.pml, fdhalf=dg.fdhalf,
                  f0_max=dg.f0_max, max_shots=len(shg), ny=dg.ny, dy=dg.dy, aniso=dg.aniso)
    g.set_model(*fg)
    pg = g.prepare(shg)
    obs = np.zeros(g.seis_size(pg), dtype=np.float32)
    go = RunOpts(checkpoint_precision=L.OWL_CKPT_FP16, checkpoint_interval=-1)
    _, gr = g.gradient(pg, obs, opts=go)
    info = g.last_info
    out["gradient_finite"] = bool(np.all(np.isfinite(np.asarray(gr))))
    out["gradient_workload"] = (f"{grad_shots} of the 16 shots, all 2500 steps, 256^3 model (296^3 padded), "
                                f"gradient w.r.t. c11, c12, c13, c22, c23, c33, c44, c55, c66, rho, FP16 checkpoints, "
                                f"L2 misfit against zero data")
    out["gradient_s_per_shot"] = info.elapsed_ms / 1e3 / len(shg)
    out["gradient_plan"] = {"shots_per_batch": info.shots_per_launch, "checkpoint_interval": info.checkpoint_interval,
                            "batches": info.batches}
    ring_a = info.tile_z == 1
    out["adjoint_kernels"] = "z-marching ring" if ring_a else "thread per cell"
    for kid, name in ((L.OWL_K_ADJ_P, "k_el3d_adj_v_ring" if ring_a else "k_el3d_adj_v"),
                      (L.OWL_K_ADJ_V, "k_el3d_adj_s_ring" if ring_a else "k_el3d_adj_s")):
        kms, b = g.kernel_time(kid, 5)
        ach = b / (kms / 1e3) / 1e9
        out["kernels"][name] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                "peak_source": peak_kind, "alg_bytes_per_launch": b, "ms_per_launch": kms,
                                "shots_per_launch": info.shots_per_launch, "model": "256^3",
                                "traffic": profile_traffic(name)}
    g.close()
    return out


# ----------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for ln in fh:
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        busy = [v for v in sm if v > 0.5 * smax] or sm
        return {"sm_mhz": busy[len(busy) // 2], "sm_max_mhz": smax, "reasons": reasons, "samples": len(rows)}


def misfit_block(s, ps, obs_dev, opts, l2_ms):
    """Each data-domain misfit on the gradient workload: the gradient of the
    32-shot batch with the misfit's adjoint source computed on the GPU, and the
    standalone adjoint-source call on the batch's gathers (device buffers)."""
    import torch
    from owl_b200 import _lib as L
    from owl_b200.solver import MisfitOpts, adjoint_source

    nt = s.desc.nt
    gp = s.gather_ptr(ps)
    syn = torch.empty(s.seis_size(ps), dtype=torch.float32, device="cuda")
    s.forward(ps, opts, out=syn)
    syn2, obs2 = syn.view(-1, nt), obs_dev.view(-1, nt)
    ntr = syn2.shape[0]
    out = {"workload": f"the gradient workload ({ps.nshots} shots); adjoint sources of its {len(gp) - 1} gathers, "
                       f"{ntr} traces of {nt} samples; adaptive: linear penalty, tlag_max 0.2 s, deconv_eps 0.1"}
    for name, kind in L.MISFIT_NAMES.items():
        if kind == L.OWL_MISFIT_DTW_VECTOR:
            continue  # one component per shot here: the same as dtw
        mo = MisfitOpts(misfit=kind, dt=s.desc.dt, tlag_max=0.2)
        if kind in (L.OWL_MISFIT_DTW, L.OWL_MISFIT_LOCAL_ADAPTIVE):
            # DTW's dynamic program costs O(nt m^2) double-precision steps per trace
            # (m = 2 tlag_max / dt + 1 = 401 candidate shifts here), the local
            # adaptive misfit five length-2 nt transforms per sample: their adjoint
            # sources are timed on the first 4 gathers, without a gradient
            g4 = gp[:5]
            n4 = int(g4[-1])
            adjoint_source(mo, g4, syn2[:n4], obs2[:n4])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            adjoint_source(mo, g4, syn2[:n4], obs2[:n4])
            ams = (time.perf_counter() - t0) * 1e3
            what = "401 candidate shifts" if kind == L.OWL_MISFIT_DTW else "Gaussian windows of 0.25 s"
            out[name] = {"sample": f"4 gathers, {n4} traces of {nt} samples, {what}",
                         "adjoint_source_ms": ams, "traces_per_s": n4 / (ams / 1e3)}
            continue
        s.gradient_misfit(ps, obs_dev, mo, opts)
        s.gradient_misfit(ps, obs_dev, mo, opts)
        gms = s.last_info.elapsed_ms
        adjoint_source(mo, gp, syn2, obs2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            adjoint_source(mo, gp, syn2, obs2)
        ams = (time.perf_counter() - t0) / 3 * 1e3
        out[name] = {"gradient_s_per_shot": gms / 1e3 / ps.nshots, "gradient_vs_l2": gms / l2_ms,
                     "adjoint_source_ms": ams, "traces_per_s": ntr / (ams / 1e3)}
    return out


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary, scaled to
    the bench's launch (None if absent)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


# ----------------------------------------------------------------------------- workload
CKPT_K = 50


def workload_config(world: int, nshots: int) -> dict:
    """The `config` of both arms' JSON lines (the same workload, whichever
    implementation runs it)."""
    return {"workload": "2D acoustic FWI gradient (L2 misfit), 201x401 grid, dx 10 m, 20-cell CFS-PML, 8th order, "
                        "dt 1 ms, 2000 steps, 32 shots per GPU (x 100..3900 m, z 20 m, 10 Hz Ricker) with receivers "
                        "every 10 m within +-1500 m offset, gradient w.r.t. (Vp, rho) with every-50-step "
                        "checkpoints",
            "shots_per_gpu": nshots, "checkpoint_interval": CKPT_K,
            "parallelism": f"shots sharded over {world} GPU(s)",
            "l2_flush": "inputs larger than L2: the 32-shot checkpoints (1.7 GB) and segment stencil terms "
                        "(2.0 GB) stream through HBM every step"}


def host_cpu_info() -> dict:
    """CPU model, physical cores and logical CPUs of this host (lscpu, else /proc/cpuinfo)."""
    info = {"logical_cpus": os.cpu_count() or 1}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        kv = {}
        for ln in out.splitlines():
            if ":" in ln:
                k, v = ln.split(":", 1)
                kv[k.strip()] = v.strip()
        info["cpu_model"] = kv.get("Model name")
        sockets = int(kv.get("Socket(s)", "0") or 0)
        cps = int(kv.get("Core(s) per socket", "0") or 0)
        if sockets and cps:
            info["physical_cores"] = sockets * cps
        info["threads_per_core"] = int(kv.get("Thread(s) per core", "0") or 0) or None
    except Exception:
        pass
    if not info.get("cpu_model"):
        try:
            with open("/proc/cpuinfo") as f:
                for ln in f:
                    if ln.startswith("model name"):
                        info["cpu_model"] = ln.split(":", 1)[1].strip()
                        break
        except Exception:
            pass
    return info


# ----------------------------------------------------------------------------- CPU baseline
_REF_CASE = None


def _ref_case():
    global _REF_CASE
    if _REF_CASE is None:
        import numpy as np
        import oracle
        from owl_b200 import configs
        from owl_b200.geometry import GridSpec, PreparedShots

        d, (vp, rho), (vp0, rho0), shots = configs.config2(NSHOTS)
        oracle.build()
        prepared = [PreparedShots([sh], GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz), d.dt) for sh in shots]
        rng = np.random.default_rng(0)
        adj = [rng.standard_normal(p.arr[0].nrec * d.nt).astype(np.float32) for p in prepared]
        _REF_CASE = (d, vp0, rho0, prepared, adj)
    return _REF_CASE


def cpu_reference_shot(i: int):
    """The reference's own gradient algorithm (restated loops: forward with
    boundary saving, -dt reconstruction, adjoint and imaging every step; OpenMP
    on the host threads) over all 2000 steps of shot i % 32 of the workload.
    Returns (seconds, threads)."""
    import oracle
    d, vp0, rho0, prepared, adj = _ref_case()
    k = i % len(prepared)
    t0 = time.perf_counter()
    oracle.ac2d_ref_gradient(d, vp0, rho0, prepared[k], adj[k], cc=1)
    el = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return el, threads


def run_reference(args, rank, world):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    _ref_case()
    secs = []
    for i in range(args.warmup + args.steps):
        el, threads = cpu_reference_shot(i)
        if i >= args.warmup:
            secs.append(el)
    v = sum(secs) / len(secs)
    sample = (f"one step = the full 2000-step gradient of one shot of the workload (shot i mod 32 at step i), "
              f"reference algorithm (forward with boundary saving, -dt reconstruction, adjoint, imaging every "
              f"step), {threads} OpenMP threads; mean of {len(secs)} shots")
    line = {
        "impl": "reference", "metric": "fwi_gradient_s_per_shot", "value": v, "unit": "s/shot",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(world, args.nshots),
        "algorithm": "the reference's time-reversed gradient (boundary saving, -dt reconstruction), restated "
                     "in C++/OpenMP (the Fortran cannot be built here), on the host CPU",
        "cpu_baseline": {"value": v, "unit": "s/shot", "cores": threads, "kind": "port", "sample": sample,
                         "host": host_cpu_info()},
        "e2e": {"value": v, "unit": "s/shot", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s_timed": sum(secs),
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm
def headline_roofline(s, d, k, peak, peak_kind):
    """Standalone CUDA-event timing of every stencil kernel variant one
    gradient launches, weighted by its launches per gradient at checkpoint
    interval k; the roofline of the one with the largest total time."""
    from owl_b200 import _lib as L
    nt = d.nt
    nseg = -(-nt // k)
    n_last = nt - (nseg - 1) * k
    # forward: all but the last segment plain, the last storing; recompute of
    # the other segments storing; adjoint every step
    counts = {L.OWL_K_FWD_P: nt - n_last, L.OWL_K_FWD_V: nt - n_last, L.OWL_K_FWD_P_STORE: nt,
              L.OWL_K_FWD_V_STORE: nt, L.OWL_K_ADJ_P: nt, L.OWL_K_ADJ_V: nt}
    # the autotuner's variants: tile codes 100 + h are the four-cell kernels,
    # 200 + h the same with the pipelined adjoint p kernel, 300 + h the
    # one-cell kernels with it (pipelined only when a CTA takes several shots)
    tzf, tza = s.last_info.tile_z_forward, s.last_info.tile_z
    v4f = 100 <= tzf < 300
    v4a = 100 <= tza < 300
    pfa = tza >= 200 and s.last_info.shots_per_cta > 1
    fp, fv = ("k_ac2d_fwd_p4", "k_ac2d_fwd_v4") if v4f else ("k_ac2d_fwd_p", "k_ac2d_fwd_v")
    ap, av = ("k_ac2d_adj_p4", "k_ac2d_adj_v4") if v4a else ("k_ac2d_adj_p", "k_ac2d_adj_v")
    if pfa:
        ap = ap + "_pf"
    names = {L.OWL_K_FWD_P: fp + "<4,0>", L.OWL_K_FWD_V: fv + "<4,0>",
             L.OWL_K_FWD_P_STORE: fp + "<4,1>", L.OWL_K_FWD_V_STORE: fv + "<4,1>",
             L.OWL_K_ADJ_P: ap + "<4>", L.OWL_K_ADJ_V: av + "<4>"}
    kt = {}
    for kid in names:
        if counts[kid] > 0:
            kt[kid] = s.kernel_time(kid, 50)
    dom = max(kt, key=lambda q: kt[q][0] * counts[q])
    ms_k, bytes_k = kt[dom]
    achieved = bytes_k / (ms_k / 1e3) / 1e9
    short = names[dom].split("<")[0]
    return {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": profile_traffic(short),
            "alg_bytes_per_launch": bytes_k, "ms_per_launch": ms_k,
            "kernel_ms_per_launch": {names[q]: kt[q][0] for q in kt},
            "launches_per_gradient": {names[q]: counts[q] for q in kt},
            "kernel_ms_per_gradient": {names[q]: kt[q][0] * counts[q] for q in kt},
            "tile_codes": {"forward": s.last_info.tile_z_forward, "adjoint": s.last_info.tile_z,
                           "shots_per_cta": s.last_info.shots_per_cta,
                           "shots_per_cta_forward": s.last_info.shots_per_cta_forward}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.profile3d:
        return profile_3d(args.profile3d, args.rows)
    if args.profile_el:
        return profile_elastic(args.profile_el, args.tile_z or 8)
    if args.profile_el3:
        return profile_elastic3(args.profile_el3, args.ring)
    if args.profile_el3_fwd:
        return profile_elastic3_forward(args.profile_el3_fwd, args.ring)
    if args.profile3d_grad:
        return profile_3d_grad(args.profile3d_grad)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from owl_b200 import _lib as L
    from owl_b200 import configs
    from owl_b200.dist import ShotSharding
    from owl_b200.solver import RunOpts, SSGSolver

    nshots = args.nshots
    d, (vp, rho), (vp0, rho0), _ = configs.config2(NSHOTS)
    # the job's shot set: nshots per GPU evenly spread over the line, sharded by trace count
    all_shots = configs.config2_shots(nshots * world, d.nx, d.dx)
    sh = ShotSharding(all_shots, rank, world)
    shots = sh.local(all_shots)
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=max(nshots, len(shots)))
    ps = s.prepare(shots)
    s.set_model(vp, rho)
    obs = s.forward(ps)  # observed data from the true model (not timed)
    s.set_model(vp0, rho0)
    opts = RunOpts(checkpoint_interval=CKPT_K)
    if args.profile and args.tile_z:
        opts = RunOpts(checkpoint_interval=CKPT_K, tile_z=args.tile_z, shots_per_cta=max(1, args.spt))
    nm = d.nx * d.nz
    obs_dev = torch.from_numpy(obs).cuda()
    g_dev = torch.zeros(2 * nm, dtype=torch.float32, device="cuda")
    m_dev = torch.zeros(len(shots), dtype=torch.float64, device="cuda")
    if args.profile:
        s.gradient(ps, obs_dev, opts=opts, grad=g_dev, misfit=m_dev)
        torch.cuda.synchronize()
        print(f"profile step: {s.last_info.elapsed_ms:.1f} ms, {s.last_info.gpu_launches} launches")
        s.close()
        return

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    red = {}

    def step_device():
        s.gradient(ps, obs_dev, opts=opts, grad=g_dev, misfit=m_dev)
        ms = s.last_info.elapsed_ms
        if world > 1:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            red["g"], red["m"] = sh.reduce(g_dev, m_dev)
            ev1.record()
            ev1.synchronize()
            ms += ev0.elapsed_time(ev1)
        return ms

    for _ in range(args.warmup):
        step_device()
    barrier()
    clk = Clocks(local)
    clk.start()
    t_wall = time.perf_counter()
    step_ms = [step_device() for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - t_wall
    clocks = clk.stop()
    launches = int(s.last_info.gpu_launches) * args.steps
    tot = torch.tensor([sum(step_ms)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    ms_step = float(tot.item()) / args.steps
    shots_job = len(all_shots)
    value = ms_step / 1e3 / shots_job
    cells = (d.nx + 2 * d.pml) * (d.nz + 2 * d.pml)
    kk = opts.checkpoint_interval
    passes = 2.0 + (-(-d.nt // kk) - 1) * kk / d.nt  # forward, recompute of all but the last segment, adjoint
    gcells = passes * cells * d.nt * shots_job / (ms_step / 1e3) / 1e9

    # e2e: the same call through the C ABI with pinned host buffers (H2D of the
    # observed data and D2H of gradient + misfit inside the timed region)
    obs_pin = torch.from_numpy(obs).pin_memory().numpy()
    g_pin = torch.zeros(2 * nm, dtype=torch.float32).pin_memory().numpy()
    m_pin = torch.zeros(len(shots), dtype=torch.float64).pin_memory().numpy()
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        s.gradient(ps, obs_pin, opts=opts, grad=g_pin, misfit=m_pin)
        ms = s.last_info.elapsed_ms
        if world > 1:
            t0 = time.perf_counter()
            gt, mt = sh.reduce(torch.from_numpy(g_pin).cuda(), torch.from_numpy(m_pin).cuda())
            gt.cpu(), mt.cpu()
            ms += (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            e2e_ms.append(ms)
    te = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = float(te.item()) / args.steps / 1e3 / shots_job

    peak, peak_kind = measured_peak_hbm()
    roofline = headline_roofline(s, d, kk, peak, peak_kind)

    line = {
        "metric": "fwi_gradient_s_per_shot", "value": value, "unit": "s/shot", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(world, nshots),
        "algorithm": "exact discrete adjoint, FP32 checkpoints every 50 steps with segment recompute (the "
                     "forward stores the last segment's stencil terms), all shots of a GPU in each stencil "
                     "launch, CUDA-graph time loop; FP64 misfit, chain rule and cross-rank reductions",
        "gcells_per_s": gcells,
        "wall_s_timed": wall,
        "e2e": {"value": e2e_value, "unit": "s/shot", "h2d_bytes_per_step": int(obs.nbytes),
                "d2h_bytes_per_step": int(g_pin.nbytes + m_pin.nbytes)},
        "gpu_launches": launches,
        "roofline": roofline,
        "clocks": clocks,
    }
    if world > 1:
        line["shots_per_rank"] = len(shots)

    extras = rank == 0 and world == 1
    if extras and not args.no_plain:
        # plain per-shot path at the same checkpoint interval: one shot per launch
        # sequence, no graphs, FP32 checkpoints
        sub = s.prepare(shots[:4])
        obs_sub = torch.from_numpy(obs[: s.seis_size(sub)]).cuda()
        po = RunOpts(checkpoint_interval=CKPT_K, shots_per_launch=1, use_graph=-1)
        s.gradient(sub, obs_sub, opts=po)
        s.gradient(sub, obs_sub, opts=po)
        line["plain_s_per_shot"] = s.last_info.elapsed_ms / 1e3 / sub.nshots
        line["batched_vs_plain"] = line["plain_s_per_shot"] / value
        line["plain_workload"] = "4 of the 32 shots, one shot per launch sequence, no CUDA graphs, every-50-step checkpoints"

    if extras:
        # the same batched gradient with the stencil terms of all 2000 steps kept in
        # HBM by the forward (~92 GB; nothing recomputed), when the device has room
        try:
            oa = RunOpts(checkpoint_interval=d.nt)
            s.gradient(ps, obs_dev, opts=oa, grad=g_dev, misfit=m_dev)
            ams = []
            for _ in range(3):
                s.gradient(ps, obs_dev, opts=oa, grad=g_dev, misfit=m_dev)
                ams.append(s.last_info.elapsed_ms)
            line["value_all_steps_stored"] = sum(ams) / len(ams) / 1e3 / len(shots)
        except L.OwlError as e:
            if e.code != L.OWL_ERR_OOM:
                raise
            line["value_all_steps_stored"] = None
        # back to the headline's buffers for the checks below
        s.gradient(ps, obs_dev, opts=opts, grad=g_dev, misfit=m_dev)

    if extras and not args.no_check:
        import oracle
        one = s.prepare(shots[:1])
        n1 = s.seis_size(one)
        _, g1 = s.gradient(one, obs[:n1].copy(), opts=opts)
        _, gref, _ = oracle.ac2d_gradient(s.desc, vp0, rho0, one, obs[:n1], adj_kind=0, k=CKPT_K, precision="f64")
        line["grad_rel_err_vs_fp64_oracle"] = float(np.linalg.norm(g1 - gref) / np.linalg.norm(gref))

    if extras:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        el, threads = cpu_reference_shot(0)
        line["cpu_baseline"] = {"value": el, "unit": "s/shot", "cores": threads, "kind": "port",
                                "sample": "shot 1 of the 32, all 2000 steps, the reference's own gradient "
                                          "algorithm (restated loops, OpenMP)", "host": host_cpu_info()}

    if extras and not args.no_misfits:
        line["misfits"] = misfit_block(s, ps, obs_dev, opts, ms_step)

    s.close()
    if extras and not args.no_3d:
        line["forward_3d"] = forward_3d_block(peak, peak_kind)
    if extras and not args.no_elastic:
        line["elastic_2d"] = elastic_2d_block(peak, peak_kind)
        line["elastic_3d"] = elastic_3d_block(peak, peak_kind, grad_shots=args.el3_grad_shots)

    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        red.clear()
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
