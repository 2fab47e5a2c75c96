#!/usr/bin/env python
"""Benchmark: TOF-TOR listmode projection + back-projection throughput (LORs/s).

Workload (default): 128x128x64 image at 3.2 mm, ring scanner R = 400 mm with
400 crystals x 32 rings (3.2 mm pitch), 10M seeded events from a cylinder phantom with
four hot spheres, TOF 530 ps FWHM (tof_sigma2 = 1139.77 mm^2, 40 ps = 6 mm bins),
TOR kernel_width 10.19 mm (FWHM 4 mm), geometry-sigma correction off. Events are
synthetic (no public dataset is involved) and preprocessed on the GPU by
``recon_process`` before the timed region.

One step = the OSEM numerator pass the reference runs per iteration
(model/recon_step.py:38-40): TOR projection of all three dominant-axis groups, then
the reference's back-projection A^T(1/Ax) of all three groups into one image (one
combined library call per group; ``--separate-ops`` makes the two calls); with
N > 1 GPUs each rank owns its own 10M events (weak scaling) and the back-projected
images are summed with one NCCL all-reduce.

* ``value``: LORs/s over all ranks with inputs resident in HBM (LOR records 400 MB per
  rank, larger than the 126 MB L2, so no flush is needed between steps).
* ``e2e``: the same metric through the public API from pinned HOST buffers: each step
  copies the raw events host->device, preprocesses them, projects, back-projects and
  copies the image back.
* ``roofline``: the dominant op's algorithmic bytes per call (per LOR: the 40-byte
  record, 4 bytes of output or value, and 4 bytes per non-zero-weight voxel sample for
  the projection, 8 for the back-projection's read-modify-write; the combined call,
  which runs both, counts both) over its CUDA-event duration inside the timed region,
  against the measured HBM copy bandwidth; plus the bound of the slowest of HBM, L2 and
  SFU (ex2) at their measured peaks.
* ``cpu_baseline``: the reference's own projector sources compiled for the host
  (oracle/_ref), all host threads, on a bounded sample of the same LORs.

``--impl reference`` times that CPU reference as the reference arm.
"""

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TOF-TOR proj+backproj LORs/s at 128x128x64 (10M events)"
METRICS = {
    "tor128": METRIC,
    "large256": "TOF-TOR proj+backproj LORs/s at 256x256x128 (16M-event chunk of the "
                "200M-event large axial FOV workload)",
    "siddon64": "non-TOF Siddon proj+backproj LORs/s at 64x64x32 (1M events)",
}
UNIT = "LORs/s"


# When set to a list, bench lines are collected there instead of printed (the default run
# embeds the other workloads' lines in its own).
_COLLECT = None


def emit(line):
    if _COLLECT is not None:
        _COLLECT.append(line)
    else:
        print(json.dumps(line), flush=True)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--events", type=int, default=None, help="override events per rank")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--workload", default="tor128",
                    choices=["tor128", "large256", "large256_recon", "siddon64", "batched96",
                             "autograd128"],
                    help="tor128: the headline TOF-TOR pair (default); large256: the same "
                         "pair on one 16M-event chunk of the large axial FOV workload "
                         "(256x256x128 at 2.5 mm, 1 m axial, 400 ps); large256_recon: that "
                         "reconstruction end to end (200M events streamed in 16M chunks, "
                         "effmap from 500M LORs, OSEM 2 x 20); siddon64: the plain "
                         "non-TOF Siddon pair and OSEM iteration (64x64x32, 1M events); "
                         "autograd128: forward + backward of 5 unrolled OSEM iterations "
                         "(128x128x64, 8 frames x 5M events); batched96: 64-frame "
                         "batched OSEM iteration vs the plain per-frame loop")
    ap.add_argument("--frames", type=int, default=64)
    ap.add_argument("--no-order", dest="order", action="store_false",
                    help="keep the preprocessed records in recon_process order, and the "
                         "effmap's map records in map_process order, instead of grouping "
                         "similar directions (preprocess.order_by_direction)")
    ap.add_argument("--separate-ops", dest="combined", action="store_false",
                    help="run projection and back-projection as two library calls (the "
                         "reference's op sequence) instead of the combined TOR call")
    ap.add_argument("--no-effmap", dest="effmap", action="store_false",
                    help="skip timing the efficiency-map pass (random detector pairs)")
    ap.add_argument("--no-variants", dest="variants", action="store_false",
                    help="skip the config variants of the same step (the reference preset "
                         "kernel_width 4.0; the geometric sigma2 factor on)")
    ap.add_argument("--effmap-source", default="tensor", choices=["generated", "tensor"],
                    help="effmap LORs: generated per chunk as a tensor, preprocessed and "
                         "ordered by direction (tensor, the default: the faster path), or "
                         "made inside the map kernels from their number with no LOR array "
                         "(generated)")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="default workload: skip the runs of the other configurations "
                         "(Siddon 64, batched 96, differentiable 128, large FOV 256) whose "
                         "summaries the line carries under 'configs'")
    ap.add_argument("--tuning", default=None,
                    help="PATH,SLAB_SLICES,GRID_MULT for srf_tor_set_tuning, or PATH for "
                         "srf_siddon_set_tuning with --workload siddon64 (default: the "
                         "library's automatic choice)")
    return ap.parse_args(argv)


def project_back(model, image, data, combined=True):
    """The step's projection then back-projection of the projected values (the reference
    recon step's numerator); ``combined`` uses the one-call TOR entry point."""
    from srf_b200 import backprojection, projection, projection_backprojection
    if combined:
        return projection_backprojection(model, image, data)[1]
    return backprojection(model, projection(model, image, data), image)


def time_variants(wl, data, image, tof_bin, tof_sigma2, combined, world, steps=5, warmup=3):
    """The timed step under the workload's variants: the reference preset's
    kernel_width 4.0 (resource/recon_task.json:46; window 3 x 3 at 3.2 mm) and the
    geometric sigma2 factor switched on (geo_sigma2_flag, the TOR sigma scaled per LOR).
    Same events, image and TOF; CUDA events, max over ranks."""
    from srf_b200 import SplitLoRsModel
    out = {}
    n = sum(data[a].lors.shape[0] for a in "xyz")
    for name, kw, geo in (("kw4", 4.0, False), ("geo", wl.kernel_width, True)):
        m = SplitLoRsModel(kw, geo, tof_sigma2=tof_sigma2, tof_bin=tof_bin)
        for _ in range(warmup):
            project_back(m, image, data, combined)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(steps):
            project_back(m, image, data, combined)
        s1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(s0.elapsed_time(s1), world) / steps
        out[name] = {"kernel_width": kw, "geo_sigma2_flag": geo, "steps": steps,
                     "ms_per_step": ms, "value": n * world / (ms / 1e3), "unit": UNIT}
    return out


def time_osem(model, data, effinv, wl, dev, warmup=1):
    """The workload's OSEM (wl.iterations x wl.subsets, records ordered inside each subset,
    eager launches) timed with CUDA events after ``warmup`` untimed iterations of another
    instance."""
    from srf_b200 import recon
    from srf_b200.preprocess import initial_image
    x0 = _image_of(initial_image(list(wl.grid), wl.center, wl.size, wl.scanner.inner_radius,
                                wl.scanner.axial_length, dev), wl)
    if warmup:
        recon.OSEM(model, data, effinv, x0, n_subsets=wl.subsets).run(warmup)
    osem = recon.OSEM(model, data, effinv, x0, n_subsets=wl.subsets)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    osem.run(wl.iterations)
    s1.record()
    torch.cuda.synchronize()
    ms = s0.elapsed_time(s1)
    n = sum(data[a].lors.shape[0] for a in "xyz")
    return {"iterations": wl.iterations, "subsets": wl.subsets, "ms": ms,
            "ms_per_iteration": ms / wl.iterations,
            "lors_per_s": n * wl.iterations / (ms / 1e3),
            "path": "recon.OSEM: per subset one combined projection + back-projection call "
                    "per axis group, then the multiplicative update"}


def _image_of(t, wl):
    from srf_b200 import Image
    return Image(t, wl.center, wl.size)


def effmap_source(args, wl, n, seed, dev):
    """The effmap's detector-pair source for ``--effmap-source``: LORs made inside the map
    kernels (``GeneratedPairs``), or generated per 16M chunk as a tensor
    (``RandomLorSource``)."""
    from srf_b200 import synthetic as S
    if args.effmap_source == "generated":
        return S.GeneratedPairs.random(wl.scanner, n, seed, device=dev)
    return S.RandomLorSource(n, wl.scanner, seed, device=dev)


def run_large_recon(args):
    """The large axial FOV reconstruction end to end: 200M seeded TOF events (400 ps) from
    the multi-cylinder phantom, streamed in 16M-event chunks from pinned host memory
    through recon_process; the efficiency map from 500M random detector pairs generated on
    the device; OSEM 2 iterations x 20 subsets at 256x256x128 (2.5 mm). Each chunk's events
    are generated on the device and copied to the pinned buffer outside the timed parts,
    standing in for a read from storage."""
    from srf_b200 import recon
    from srf_b200 import preprocess as PP
    from srf_b200 import synthetic as S
    from srf_b200.preprocess import initial_image
    from srf_b200.scanner import tof_info
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    wl = S.large_256()
    n_total = args.events or wl.n_events
    chunk = 16_000_000
    tof_bin, tof_sigma2 = tof_info(wl.tof_res_ps, wl.tof_bin_ps)
    model = model_for(wl, tof_bin, tof_sigma2)
    phantom = S.large_fov_phantom(half_length=wl.scanner.axial_length / 2)
    host = torch.empty((min(chunk, n_total), 7), dtype=torch.float32).pin_memory()
    dbuf = torch.empty((min(chunk, n_total), 7), dtype=torch.float32, device=dev)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        return r, a.elapsed_time(b)

    parts, stream_ms, gen_s = {a: [] for a in "xyz"}, 0.0, 0.0
    for k, start in enumerate(range(0, n_total, chunk)):
        c = min(chunk, n_total - start)
        t0 = time.perf_counter()
        ev = S.generate_events(c, wl.scanner, phantom, seed=wl.seed * 1000 + k,
                               tof_sigma_mm=math.sqrt(tof_sigma2), device=dev)
        host[:c].copy_(ev)
        del ev
        gen_s += time.perf_counter() - t0

        def upload_and_preprocess():
            dbuf[:c].copy_(host[:c], non_blocking=True)
            return PP.recon_process(dbuf[:c], wl.tof_res_ps)

        g, ms = timed(upload_and_preprocess)
        stream_ms += ms
        for a in "xyz":
            parts[a].append(g[a])
    groups = {a: torch.cat(v) for a, v in parts.items()}
    del parts
    data = PP.split_listmode(groups)
    args_e = (list(wl.grid), wl.center, wl.size, wl.scanner.inner_radius,
              wl.scanner.axial_length)
    recon.efficiency_map(model, effmap_source(args, wl, chunk, 78, dev), *args_e,
                         order=args.order)  # warm-up: one chunk (sizes the scratch pool)
    (effinv, _), effmap_ms = timed(lambda: recon.efficiency_map(
        model, effmap_source(args, wl, wl.n_effmap, 77, dev), *args_e, order=args.order))
    x0 = _image_of(initial_image(list(wl.grid), wl.center, wl.size, wl.scanner.inner_radius,
                                 wl.scanner.axial_length, dev), wl)
    osem, setup_ms = timed(lambda: recon.OSEM(model, data, effinv, x0, n_subsets=wl.subsets))
    del data, groups
    _, osem_ms = timed(lambda: osem.run(wl.iterations))
    total_ms = stream_ms + effmap_ms + setup_ms + osem_ms
    x = osem.x.data
    line = {"metric": "large axial FOV TOF OSEM end to end (256x256x128, 200M events in "
                      "16M-event chunks, 2 it x 20 subsets, effmap from 500M random LORs)",
            "value": total_ms / 1e3, "unit": "s", "higher_is_better": False, "n_gpus": 1,
            "events": n_total, "stream_preprocess_ms": stream_ms, "effmap_ms": effmap_ms,
            "osem_setup_ms": setup_ms, "osem_ms": osem_ms,
            "osem_lors_per_s": n_total * wl.iterations / (osem_ms / 1e3),
            "effmap_lors_per_s": wl.n_effmap / (effmap_ms / 1e3),
            "image_finite": bool(torch.isfinite(x).all()), "image_sum": float(x.sum()),
            "generation_s_untimed": gen_s, "dtype": "f32",
            "data": "synthetic (seeded events from the multi-cylinder phantom)",
            "config": {"workload": "large_256x256x128_200M_recon", "grid": list(wl.grid),
                       "voxel_mm": wl.voxel, "tof_res_ps": wl.tof_res_ps,
                       "kernel_width": round(wl.kernel_width, 4), "chunk_events": chunk,
                       "iterations": wl.iterations, "subsets": wl.subsets,
                       "effmap_lors": wl.n_effmap, "effmap_source": args.effmap_source},
            "path": "per chunk: pinned host events -> device -> recon_process; effmap: "
                    "on-device random pairs -> map_process -> maplors; OSEM: subsets split "
                    "and ordered once, then per subset one combined projection + "
                    "back-projection call per axis group and the update"}
    emit(line)
    return 0


# ------------------------------------------------------------------ distributed


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pipelined_e2e(host_events, compute, steps, dev):
    """Device ms of ``steps`` end-to-end steps. Step k copies its events from pinned host
    memory into one of two device buffers, runs ``compute(events) -> device image`` and
    copies the image back into pinned host memory. The copy of step k+1's events runs on a
    second stream while step k computes; each step still moves its own inputs and result
    across the host link inside the timed region."""
    main = torch.cuda.current_stream(dev)
    cs = torch.cuda.Stream(device=dev)
    bufs = [torch.empty(host_events.shape, dtype=host_events.dtype, device=dev)
            for _ in range(2)]
    up = [torch.cuda.Event() for _ in range(2)]
    out_host = None

    def upload(k):
        b = k % 2
        cs.wait_stream(main)  # step k-2, the buffer's last user, is enqueued before this
        with torch.cuda.stream(cs):
            bufs[b].copy_(host_events, non_blocking=True)
            up[b].record(cs)

    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(main)
    upload(0)
    for k in range(steps):
        main.wait_event(up[k % 2])
        if k + 1 < steps:
            upload(k + 1)
        img = compute(bufs[k % 2])
        if out_host is None:
            out_host = torch.empty(img.shape, dtype=img.dtype).pin_memory()
        out_host.copy_(img, non_blocking=True)
    s1.record(main)
    torch.cuda.synchronize(dev)
    return s0.elapsed_time(s1)


# ----------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi sampling of the SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # the timed region starts once sampling runs (nvidia-smi takes a moment)
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, flags in rows for k, f in enumerate(flags)
                          if f.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


# --------------------------------------------------------------------- workload


def workload_inputs(events_per_rank, rank, device, name="tor128"):
    from srf_b200 import synthetic as S
    from srf_b200.scanner import tof_info
    wl = S.large_256() if name == "large256" else S.tor_128()
    chunk = 16_000_000 if name == "large256" else wl.n_events  # large FOV: streamed chunks
    n = events_per_rank or chunk
    tof_bin, tof_sigma2 = tof_info(wl.tof_res_ps, wl.tof_bin_ps)
    if name == "large256":
        phantom = S.large_fov_phantom(half_length=wl.scanner.axial_length / 2)
    else:
        phantom = S.standard_phantom(half_length=wl.scanner.axial_length / 2)
    events = S.generate_events(n, wl.scanner, phantom, seed=wl.seed + 7919 * rank,
                               tof_sigma_mm=math.sqrt(tof_sigma2), device=device)
    img = phantom.voxelize(wl.grid, wl.center, wl.size) + np.float32(0.05)
    return wl, events, img, tof_bin, tof_sigma2


def model_for(wl, tof_bin, tof_sigma2):
    from srf_b200 import SplitLoRsModel
    return SplitLoRsModel(wl.kernel_width, False, tof_sigma2=tof_sigma2, tof_bin=tof_bin)


def algorithmic_work(model, data, image):
    """Useful samples per group (voxels with non-zero weight), from the library's own
    counting kernel, and LOR counts."""
    from srf_b200 import ops
    per = {}
    for a in model.AXIS:
        _, g, c, s = model.kernel_geometry(image, a)
        cnt = ops.tor_count_samples(data[a].lors, g, c, s, model.kernel_width,
                                    model.geo_sigma2_flag, layout="nc")
        per[a] = {"lors": int(cnt.shape[1]), "useful": int(cnt[0].sum(dtype=torch.int64)),
                  "slots": int(cnt[1].sum(dtype=torch.int64))}
    return per


OPS_OF = {"srf_tor_projection": ("proj",), "srf_tor_backprojection": ("back",),
          "srf_tor_projection_backprojection": ("proj", "back")}


def roofline_components(kernel, ms_per_step, n_lors, n_groups, rec, useful, slots, image_bytes,
                        hbm_peak, probe):
    """Bound time T* of the dominant op per step, as the survey's measurement section
    defines it, T* = max(B_HBM / HBM peak, B / L2 peak, exps / SFU peak):

    * B_HBM: the bytes that must cross HBM: each LOR record (``rec`` bytes) and its value
      (4 B: the projection's output, the back-projection's input) once per op, the image
      of each axis group once per op (read by the projection, read-modify-written by the
      back-projection);
    * B: B_HBM plus the voxel samples: 4 B per useful (non-zero-weight) sample read by
      the projection, 8 B per useful sample read-modify-written by the back-projection;
    * exps: one per useful sample and op;

    each against its measured peak (HBM copy; L2 read, ex2 and shared-memory probes run
    in the same process); frac = T* / T. The slab kernels serve their samples from shared
    memory, so two shared-memory terms are reported beside the survey's three: sample
    bytes / measured shared read bandwidth, and back-projected samples / measured
    shared-memory atomicAdd rate at hashed addresses."""
    ops_ = OPS_OF.get(kernel, ("proj",))
    b_hbm = b_samp = 0
    n_atom = 0
    for op in ops_:
        b_hbm += n_lors * (rec + 4) + n_groups * image_bytes * (1 if op == "proj" else 2)
        b_samp += useful * (4 if op == "proj" else 8)
        n_atom += useful if op == "back" else 0
    exps = useful * len(ops_)
    t_meas = ms_per_step / 1e3
    terms = {
        "hbm": (b_hbm / (hbm_peak * 1e9), {"bytes": b_hbm, "peak_gbs": hbm_peak}),
        "l2": ((b_hbm + b_samp) / (probe["l2_gbs"] * 1e9),
               {"bytes": b_hbm + b_samp, "peak_gbs": probe["l2_gbs"]}),
        "sfu": (exps / probe["ex2_per_s"], {"exps": exps, "peak_ex2_per_s": probe["ex2_per_s"],
                                            "reference_exps": (useful + slots) * len(ops_)}),
    }
    side = {
        "smem_read": (b_samp / (probe["smem_gbs"] * 1e9),
                      {"bytes": b_samp, "peak_gbs": probe["smem_gbs"]}),
        "smem_atomic": (n_atom / probe["smem_atomic_random_per_s"],
                        {"atomics": n_atom,
                         "peak_per_s": probe["smem_atomic_random_per_s"],
                         "peak_per_s_conflict_free": probe["smem_atomic_per_s"]}),
    }
    out = {}
    for k, (t, extra) in list(terms.items()) + list(side.items()):
        out[k] = dict(ms=t * 1e3, frac=t / t_meas, **extra)
    bound_term = max(terms, key=lambda k: terms[k][0])
    bound = terms[bound_term][0]
    out.update({"bound_term": bound_term, "bound_ms": bound * 1e3, "measured_ms": ms_per_step,
                "frac_of_bound": bound / t_meas, "b_hbm": b_hbm, "b_total": b_hbm + b_samp,
                "probe": probe["method"]})
    return out


def roofline(kern, steps, n_lors, n_groups, useful, slots, image_bytes, hbm_peak, peak_src,
             workload):
    """The line's ``roofline`` object for the dominant op (most device time in the timed
    region): its bound T* (``roofline_components``) expressed in the binding term's units
    (``achieved`` = that term's bytes, or exps, per launch / the launch's mean CUDA-event
    time; ``frac`` = achieved / peak = T* / T), the other terms, and ``traffic``, the
    DRAM bytes per launch ncu measured for this workload (profiles/roofline_traffic.txt)."""
    from srf_b200 import profiling
    if not kern:
        return None
    dom = max(kern, key=lambda k: kern[k]["total_ms"])
    launches = kern[dom]["launches"]
    comp = roofline_components(dom, kern[dom]["total_ms"] / steps, n_lors, n_groups, 40,
                               useful, slots, image_bytes, hbm_peak, profiling.measure_peaks())
    term = comp["bound_term"]
    per_launch = steps / max(launches, 1)
    mean_s = kern[dom]["mean_ms"] / 1e3
    if term == "sfu":
        achieved = comp["sfu"]["exps"] * per_launch / mean_s / 1e12
        peak, unit = comp["sfu"]["peak_ex2_per_s"] / 1e12, "Texp/s"
    else:
        achieved = comp[term]["bytes"] * per_launch / mean_s / 1e9
        peak, unit = comp[term]["peak_gbs"], "GB/s"
    traffic = None
    prof = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if os.path.exists(prof):  # measured per workload; null where not captured
        traffic = json.load(open(prof)).get(workload, {}).get(dom)
    return {"kernel": dom, "bound": term, "achieved": achieved, "peak": peak, "unit": unit,
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": f"{peak_src} hbm_gbs (burst copy) for the HBM term; L2, ex2 and "
                           "shared-memory peaks from the library's probes in this run",
            "b_hbm_per_launch": comp["b_hbm"] * per_launch,
            "algorithmic_bytes_per_launch": comp["b_total"] * per_launch,
            "useful_samples_per_step": useful, "window_samples_per_step": slots,
            "components": comp,
            "kernel_ms": {k: {"launches": v["launches"], "mean_ms": v["mean_ms"],
                              "share": v["total_ms"] / sum(x["total_ms"] for x in kern.values())}
                          for k, v in kern.items()}}


# ------------------------------------------------------------------ CPU baseline


def host_cpu():
    """The host the CPU baseline runs on: lscpu's model name, core and thread counts and
    clock (current and maximum MHz), /proc/cpuinfo when lscpu is absent."""
    info = {"nproc": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        want = {"Model name": "model", "CPU(s)": "cpus", "Thread(s) per core": "threads_per_core",
                "Core(s) per socket": "cores_per_socket", "Socket(s)": "sockets",
                "CPU MHz": "mhz", "CPU max MHz": "max_mhz"}
        for ln in out.splitlines():
            k, _, v = ln.partition(":")
            if k.strip() in want:
                info[want[k.strip()]] = v.strip()
    except (OSError, subprocess.SubprocessError):
        pass
    if "model" not in info or "mhz" not in info:
        try:
            for ln in open("/proc/cpuinfo"):
                k, _, v = ln.partition(":")
                if k.strip() == "model name":
                    info.setdefault("model", v.strip())
                elif k.strip() == "cpu MHz":
                    info.setdefault("mhz", v.strip())
        except OSError:
            pass
    return info


def cpu_baseline(groups_host, wl, tof_bin, tof_sigma2, image_np, target_s):
    """Time the reference's host-built projector pair on a bounded sample of the same
    LORs with all host threads (oracle/_ref), falling back to the single-thread oracle
    port. Returns the cpu_baseline object."""
    from oracle import preprocess_ref as P
    from oracle import pyoracle as O
    ncpu = os.cpu_count() or 1
    if O.ReferenceHost.available():
        R = O.ReferenceHost()
        kind, threads = "reference", ncpu

        def pair(lors, img, g, c, s):
            pv = R.tor_projection(lors, img, g, c, s, wl.kernel_width, False, tof_bin,
                                  tof_sigma2, nthreads=threads)
            R.tor_backprojection(lors, pv, g, c, s, wl.kernel_width, False, tof_bin,
                                 tof_sigma2, nthreads=threads)
    else:
        kind, threads = "port", 1

        def pair(lors, img, g, c, s):
            pv = O.tor_projection(lors, img, g, c, s, wl.kernel_width, False, tof_bin,
                                  tof_sigma2, mode="f32")
            O.tor_backprojection(lors, pv, g, c, s, wl.kernel_width, False, tof_bin,
                                 tof_sigma2, mode="f32")

    views = {a: P.axis_view(image_np, wl.center, wl.size, a) for a in "xyz"}
    total = sum(groups_host[a].shape[0] for a in "xyz")

    def run(frac):
        n_done, t0 = 0, time.perf_counter()
        for a in "xyz":
            k = max(1, int(groups_host[a].shape[0] * frac))
            lors = np.ascontiguousarray(groups_host[a][:k].T)
            img, g, c, s = views[a]
            pair(lors, img, g, c, s)
            n_done += k
        return n_done, time.perf_counter() - t0

    n0, t0 = run(2000.0 / total)  # calibration
    frac = min(1.0, (2000.0 / total) * max(1.0, target_s / max(t0, 1e-3)))
    n1, t1 = run(frac)
    return {"value": n1 / t1, "unit": UNIT, "cores": threads, "kind": kind, "host": host_cpu(),
            "sample": f"{n1} LORs (first {frac * 100:.2f}% of each dominant-axis group of the "
                      f"same preprocessed events), projection + back-projection, "
                      f"{t1:.1f} s wall"}


def siddon_roofline(kern, steps, n_rays, visits, image_bytes, hbm_peak, peak_src, workload):
    """The Siddon line's ``roofline`` object for the dominant op, with the bound of the
    survey's measurement section, T* = max(B_HBM / HBM peak, B / L2 peak, exps / SFU
    peak): B_HBM = the 28 B ray record and its 4 B value or output once per ray, plus the
    image once (projection) or read-modify-written once (back-projection); B = B_HBM plus
    4 B (projection) or 8 B (back-projection) per visited voxel, served by the L2 where
    the image stays; no exps with TOF off. ``achieved`` = the binding term's bytes per
    launch / the launch's mean CUDA-event time."""
    from srf_b200 import profiling
    if not kern:
        return None
    dom = max(kern, key=lambda k: kern[k]["total_ms"])
    back = dom != "srf_siddon_projection"
    b_hbm = n_rays * 32 + image_bytes * (2 if back else 1)
    b_all = b_hbm + visits * (8 if back else 4)
    probe = profiling.measure_peaks()
    t_meas = kern[dom]["total_ms"] / steps / 1e3
    terms = {"hbm": b_hbm / (hbm_peak * 1e9), "l2": b_all / (probe["l2_gbs"] * 1e9), "sfu": 0.0}
    term = max(terms, key=terms.get)
    per_launch = steps / max(kern[dom]["launches"], 1)
    mean_s = kern[dom]["mean_ms"] / 1e3
    nbytes = (b_all if term == "l2" else b_hbm) * per_launch
    peak = probe["l2_gbs"] if term == "l2" else hbm_peak
    achieved = nbytes / mean_s / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if os.path.exists(prof):
        traffic = json.load(open(prof)).get(workload, {}).get(dom)
    return {"kernel": dom, "bound": term, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": f"{peak_src} hbm_gbs (burst copy) for the HBM term; L2 peak from "
                           "the library's probe in this run",
            "b_hbm_per_launch": b_hbm * per_launch, "algorithmic_bytes_per_launch": b_all * per_launch,
            "visited_voxels_per_step": visits,
            "components": {"hbm": {"ms": terms["hbm"] * 1e3, "frac": terms["hbm"] / t_meas,
                                   "bytes": b_hbm, "peak_gbs": hbm_peak},
                           "l2": {"ms": terms["l2"] * 1e3, "frac": terms["l2"] / t_meas,
                                  "bytes": b_all, "peak_gbs": probe["l2_gbs"]},
                           "sfu": {"ms": 0.0, "frac": 0.0, "exps": 0},
                           "bound_term": term, "bound_ms": terms[term] * 1e3,
                           "measured_ms": t_meas * 1e3, "frac_of_bound": terms[term] / t_meas},
            "kernel_ms": {k: {"launches": v["launches"], "mean_ms": v["mean_ms"],
                              "share": v["total_ms"] / sum(x["total_ms"] for x in kern.values())}
                          for k, v in kern.items()}}


def run_siddon(args):
    """Plain non-TOF Siddon (the CPU-runnable configuration): R 400 mm, 400 x 32
    crystals, 64x64x32 image at 3.4 mm, 1M seeded events from the cylinder phantom,
    tof_sigma2 = 1e6 (at or above the reference's TOF switch, so TOF is off). One step =
    Siddon projection of all events, then the reference back-projection A^T(1/Ax). Also
    times one OSEM iteration (4 subsets, effmap from 10M random crystal pairs) and the
    reference's host-built Siddon pair on a bounded sample."""
    from srf_b200 import CompleteLoRsModel, Image, ops, profiling
    from srf_b200 import recon
    from srf_b200 import synthetic as S
    from srf_b200 import _lib
    from srf_b200.data import ListModeData
    from srf_b200.preprocess import initial_image
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    if args.tuning:
        from srf_b200 import tuning
        tuning.set_siddon_tuning(int(args.tuning.split(",")[0]))
    wl = S.siddon_64()
    n = args.events or wl.n_events
    phantom = S.standard_phantom(half_length=wl.scanner.axial_length / 2)
    events = S.generate_events(n, wl.scanner, phantom, seed=wl.seed + 7919 * rank, device=dev)
    img_np = phantom.voxelize(wl.grid, wl.center, wl.size) + np.float32(0.05)
    image = Image(torch.as_tensor(img_np, device=dev), wl.center, wl.size)
    model = CompleteLoRsModel(tof_sigma2=1.0e6, tof_bin=1.0e4)
    kimg, g, c, sz = model.kernel_geometry(image)
    events_in = events  # generation order: the CPU baseline samples its head
    if args.order:
        from srf_b200.preprocess import order_rays_by_length
        events = order_rays_by_length(events, g, c, sz)
    data = ListModeData(events, torch.ones(events.shape[0], device=dev))
    visits = int(ops.siddon_count_samples(events, g, c, sz, layout="nc").sum(dtype=torch.int64))

    def step():
        bp = project_back(model, image, data, args.combined)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(bp.data)
        return bp

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if clocks:
        clocks.start()
    timer = profiling.KernelTimer()
    launches0 = _lib.call_raw("srf_launch_count")
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("bench_timed")
    with timer:
        start.record()
        for _ in range(args.steps):
            step()
        end.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier(world)
    gpu_launches = _lib.call_raw("srf_launch_count") - launches0
    ms = max_over_ranks(start.elapsed_time(end), world)
    clk = clocks.stop() if clocks else None
    kern = timer.summary()
    value = n * world * args.steps / (ms / 1e3)

    # e2e through the public API from pinned host events
    e2e = None
    if args.e2e_steps > 0:
        host_events = events.cpu().pin_memory()

        def compute(ev):
            d = ListModeData(ev, torch.ones(ev.shape[0], device=dev))
            bp = project_back(model, image, d, args.combined)
            if world > 1:
                import torch.distributed as dist
                dist.all_reduce(bp.data)
            return bp.data

        pipelined_e2e(host_events, compute, 1, dev)  # warm-up
        barrier(world)
        e_ms = max_over_ranks(pipelined_e2e(host_events, compute, args.e2e_steps, dev), world)
        e2e = {"value": n * world * args.e2e_steps / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": host_events.numel() * 4,
               "d2h_bytes_per_step": int(np.prod(wl.grid)) * 4,
               "ms_per_step": e_ms / args.e2e_steps,
               "path": "pinned host events -> projection -> backprojection -> pinned host "
                       "image; step k+1's upload overlaps step k"}

    # one OSEM iteration (4 subsets) with the effmap of 10M random crystal pairs
    lors = S.random_lors(10_000_000, wl.scanner, 77, device=dev)
    effinv, _ = recon.efficiency_map(model, lors, list(wl.grid), wl.center, wl.size,
                                     wl.scanner.inner_radius, wl.scanner.axial_length)
    del lors
    x0 = initial_image(list(wl.grid), wl.center, wl.size, wl.scanner.inner_radius,
                       wl.scanner.axial_length, dev)
    osem = recon.OSEM(model, data, effinv, Image(x0, wl.center, wl.size), n_subsets=wl.subsets)
    osem.step()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(wl.iterations):
        osem.step()
    s1.record()
    torch.cuda.synchronize()
    osem_ms = s0.elapsed_time(s1) / wl.iterations

    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    roof = siddon_roofline(kern, args.steps, n, visits, int(np.prod(wl.grid)) * 4, hbm_peak,
                           "measured" if "hbm_gbs" in peaks else "fallback", wl.name)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = siddon_cpu_baseline(events_in, model, image, args.cpu_seconds)
        except Exception as exc:  # reported, never fatal for the GPU number
            base = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                    "sample": f"unavailable: {exc}"}
    if rank == 0:
        line = {"metric": METRICS["siddon64"], "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded events from a cylinder phantom)",
                "config": {"workload": wl.name, "grid": list(wl.grid), "voxel_mm": wl.voxel,
                           "events_per_rank": int(n), "tof_sigma2": 1.0e6,
                           "parallelism": f"events sharded, {world} rank(s)",
                           "l2": "image (0.5 MB) L2-resident; LOR records 28 MB per rank",
                           "tuning": args.tuning or "automatic"},
                "osem_iteration_ms": osem_ms,
                "osem": {"subsets": wl.subsets, "iterations_timed": wl.iterations,
                         "effmap_lors": 10_000_000},
                "roofline": roof, "cpu_baseline": base, "e2e": e2e,
                "gpu_launches": gpu_launches, "clocks": clk}
        emit(line)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def siddon_cpu_baseline(events, model, image, target_s):
    """The reference's host-built Siddon pair on all host threads over a bounded sample of
    the same events. Rays the walk does not visit (they miss the image, or would make the
    reference read outside it) are counted but not run: the reference returns 0 for them."""
    from oracle import pyoracle as O
    if not O.ReferenceHost.available():
        raise RuntimeError("reference host build not present")
    R = O.ReferenceHost()
    threads = os.cpu_count() or 1
    kimg, g, c, s = model.kernel_geometry(image)
    img = kimg.cpu().numpy()
    ev = events.cpu().numpy()
    visits, _ = O.siddon_counts(np.ascontiguousarray(ev.T), g, c, s)

    def run(k):
        sel = np.ascontiguousarray(ev[:k][visits[:k] > 0].T)
        t0 = time.perf_counter()
        pv = R.siddon_projection(sel, img, g, c, s, model.tof_bin, model.tof_sigma2,
                                 nthreads=threads)
        R.siddon_backprojection(sel, pv, g, c, s, model.tof_bin, model.tof_sigma2,
                                nthreads=threads)
        return time.perf_counter() - t0

    k = min(len(ev), 20000)
    t = run(k)
    k = int(min(len(ev), k * max(1.0, target_s / max(t, 1e-3))))
    t = run(k)
    return {"value": k / t, "unit": UNIT, "cores": threads, "kind": "reference",
            "host": host_cpu(),
            "sample": f"first {k} events ({int((visits[:k] > 0).sum())} visit the image), "
                      f"projection + back-projection, {t:.1f} s wall"}


def run_autograd(args):
    """Differentiable projector at full size: 128x128x64 (3.2 mm), 8 frames of 5M events
    (TOF 530 ps). Per frame, loss = sum_i ((A x_5)_i - log (A x_5)_i) + 0.01/2 * quadratic
    6-neighbour penalty of x_5, with x_5 five unrolled MLEM iterations of x0 under
    torch.utils.checkpoint; timed: forward + backward (gradient w.r.t. x0) of all frames.
    Also the adjoint identity <A x, y> = <x, A^T y> of the autograd pair at this size."""
    from srf_b200 import Image, SplitLoRsModel
    from srf_b200 import preprocess as PP
    from srf_b200 import synthetic as S
    from srf_b200.autograd import Projector, poisson_nll, quadratic_penalty, unrolled_osem
    from srf_b200.scanner import tof_info
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    wl = S.tor_128()
    b, s2 = tof_info(wl.tof_res_ps, wl.tof_bin_ps)
    model = SplitLoRsModel(wl.kernel_width, False, tof_sigma2=s2, tof_bin=b)
    n_frames, n_ev = max(1, args.frames if args.frames != 64 else 8), args.events or 5_000_000
    projs = []
    for f in range(n_frames):
        ph = S.random_phantom(4000 + f, wl.scanner.axial_length / 2)
        ev = S.generate_events(n_ev, wl.scanner, ph, seed=4000 + f,
                               tof_sigma_mm=math.sqrt(s2), device=dev)
        data = PP.split_listmode(PP.recon_process(ev, wl.tof_res_ps))
        projs.append(Projector(model, data, list(wl.grid), wl.center, wl.size))
        del ev
    x0 = (torch.rand(wl.grid, device=dev) + 0.5).requires_grad_(True)
    effinv = torch.rand(wl.grid, device=dev) + 0.5

    def step():
        x0.grad = None
        total = 0.0
        for A in projs:
            xk = unrolled_osem(A, x0, effinv, n_iterations=5, checkpoint=True)
            loss = poisson_nll(A.forward(xk), per_event=True) + quadratic_penalty(xk, 0.01)
            loss.backward()
            total += float(loss.detach())
        return total

    step()  # warm-up
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    steps = max(1, args.steps // 5)
    for _ in range(steps):
        step()
    s1.record()
    torch.cuda.synchronize()
    ms = s0.elapsed_time(s1) / steps
    finite = bool(torch.isfinite(x0.grad).all())

    # adjoint identity of the autograd pair on the first frame at full size
    A = projs[0]
    with torch.no_grad():
        x = torch.rand(wl.grid, device=dev, dtype=torch.float32)
        p = A.forward(x)
        y = {a: torch.rand_like(v) for a, v in p.items()}
        lhs = sum(float((p[a].double() * y[a].double()).sum()) for a in p)
        rhs = float((x.double() * A.adjoint(y).double()).sum())
    line = {"metric": "differentiable unrolled OSEM forward+backward time (128x128x64, "
                      f"{n_frames} frames x {n_ev // 10**6}M events, 5 iterations)",
            "value": ms, "unit": "ms", "higher_is_better": False, "n_gpus": 1,
            "steps": steps, "frames": n_frames, "events_per_frame": n_ev,
            "adjoint_identity_rel_err": abs(lhs - rhs) / abs(lhs), "gradient_finite": finite,
            "data": "synthetic (seeded per-frame phantoms)",
            "config": {"workload": "autograd_128x128x64_8x5M", "grid": list(wl.grid),
                       "voxel_mm": wl.voxel, "checkpoint": True, "beta": 0.01}}
    emit(line)
    return 0


# ------------------------------------------------------------------ reference arm


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import preprocess_ref as P
    from srf_b200 import synthetic as S
    from srf_b200.scanner import tof_info
    wl = S.tor_128()
    tof_bin, tof_sigma2 = tof_info(wl.tof_res_ps, wl.tof_bin_ps)
    phantom = S.standard_phantom(half_length=wl.scanner.axial_length / 2)
    n_gen = 400_000
    ev = S.generate_events(n_gen, wl.scanner, phantom, seed=wl.seed,
                           tof_sigma_mm=math.sqrt(tof_sigma2)).numpy()
    groups = P.recon_process(ev, wl.tof_res_ps)
    img = phantom.voxelize(wl.grid, wl.center, wl.size) + np.float32(0.05)
    base = cpu_baseline(groups, wl, tof_bin, tof_sigma2, img, target_s=2.0)
    # each step: the same bounded sample size that calibration chose
    n_per_step = int(base["sample"].split()[0])
    frac = n_per_step / sum(groups[a].shape[0] for a in "xyz")
    from oracle import pyoracle as O
    views = {a: P.axis_view(img, wl.center, wl.size, a) for a in "xyz"}
    use_ref = O.ReferenceHost.available()
    R = O.ReferenceHost() if use_ref else None
    threads = os.cpu_count() if use_ref else 1

    def step():
        n = 0
        for a in "xyz":
            k = max(1, int(groups[a].shape[0] * frac))
            lors = np.ascontiguousarray(groups[a][:k].T)
            im, g, c, s = views[a]
            if use_ref:
                pv = R.tor_projection(lors, im, g, c, s, wl.kernel_width, False, tof_bin,
                                      tof_sigma2, nthreads=threads)
                R.tor_backprojection(lors, pv, g, c, s, wl.kernel_width, False, tof_bin,
                                     tof_sigma2, nthreads=threads)
            else:
                pv = O.tor_projection(lors, im, g, c, s, wl.kernel_width, False, tof_bin,
                                      tof_sigma2)
                O.tor_backprojection(lors, pv, g, c, s, wl.kernel_width, False, tof_bin,
                                     tof_sigma2)
            n += k
        return n

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    n = sum(step() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    value = n / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded events)", "impl": "reference",
            "config": {"workload": wl.name, "grid": list(wl.grid), "voxel_mm": wl.voxel,
                       "kernel_width": wl.kernel_width, "tof_res_ps": wl.tof_res_ps,
                       "sample_lors_per_step": n // args.steps},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                             "kind": "reference" if use_ref else "port", "host": host_cpu(),
                             "sample": f"{n // args.steps} LORs per step from the same "
                                       f"preprocessed events"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    emit(line)
    return 0


# ------------------------------------------------------------------------- ours


def run_batched(args):
    """64 independent TOF-TOR reconstructions at 96x96x48 (3.2 mm): per-frame phantom
    radius U(60,150) mm with four hot spheres, event counts log-uniform in [0.2M, 5M],
    OSEM with 10 subsets. Times one iteration of the batched OSEM (one launch per kernel
    per subset for all frames, autotuned, CUDA-graph replay) against one iteration of the
    plain per-frame loop (srf_b200.recon.OSEM per frame), and compares the images."""
    from srf_b200 import Image, SplitLoRsModel, recon, tuning
    from srf_b200 import preprocess as PP
    from srf_b200 import synthetic as S
    from srf_b200.batched import BatchedOSEM
    from srf_b200.scanner import tof_info
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    wl0 = S.batched_96(0)
    tof_bin, tof_sigma2 = tof_info(wl0.tof_res_ps, wl0.tof_bin_ps)
    model = SplitLoRsModel(wl0.kernel_width, False, tof_sigma2=tof_sigma2, tof_bin=tof_bin)
    frames, n_events = [], 0
    t0 = time.perf_counter()
    for f in range(args.frames):
        wl = S.batched_96(f)
        ph = S.random_phantom(wl.seed, wl.scanner.axial_length / 2)
        ev = S.generate_events(wl.n_events, wl.scanner, ph, seed=wl.seed,
                               tof_sigma_mm=math.sqrt(tof_sigma2), device=dev)
        frames.append(PP.recon_process(ev, wl.tof_res_ps))
        n_events += wl.n_events
        del ev
    gen_s = time.perf_counter() - t0
    grid, center, size = list(wl0.grid), wl0.center, wl0.size
    lors = S.random_lors(10_000_000, wl0.scanner, 77, device=dev)
    effinv, _ = recon.efficiency_map(model, lors, grid, center, size, wl0.scanner.inner_radius,
                                     wl0.scanner.axial_length)
    del lors
    x0 = PP.initial_image(grid, center, size, wl0.scanner.inner_radius,
                          wl0.scanner.axial_length, dev)
    S_sub = wl0.subsets

    bat = BatchedOSEM(model, frames, effinv, x0, n_subsets=S_sub)
    tuner = tuning.Autotuner()
    probe = BatchedOSEM(model, frames, effinv, x0, n_subsets=S_sub)
    best, timings = tuner.tune("batched96", lambda: probe._subset_update(0),
                               tuning.candidates(16))
    del probe
    bat.use_graph = True
    bat.step()  # capture + first iteration
    torch.cuda.synchronize()
    reps = max(1, args.steps // 5)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(reps):
        bat.step()
    s1.record()
    torch.cuda.synchronize()
    batched_ms = s0.elapsed_time(s1) / reps

    # the plain per-frame loop at its faster setting (records ordered or not)
    plain_by_order = {}
    for order in (True, False):
        plain = [recon.OSEM(model, PP.split_listmode(g), effinv, Image(x0, center, size),
                            n_subsets=S_sub, order=order) for g in frames]
        for o in plain:
            o.step()
        torch.cuda.synchronize()
        s0.record()
        for _ in range(reps):
            for o in plain:
                o.step()
        s1.record()
        torch.cuda.synchronize()
        plain_by_order[order] = (s0.elapsed_time(s1) / reps, plain)
    plain_order = min(plain_by_order, key=lambda k: plain_by_order[k][0])
    plain_ms, plain = plain_by_order[plain_order]
    errs = []
    for f, o in enumerate(plain):
        a, b = bat.x[f].double(), o.x.data.double()
        errs.append(float((a - b).norm() / b.norm()))
    tuning.set_tuning()
    line = {"metric": "batched 64-frame TOF OSEM iteration time (96x96x48, 10 subsets)",
            "value": batched_ms, "unit": "ms", "higher_is_better": False, "n_gpus": 1,
            "plain_loop_ms": plain_ms, "speedup_vs_plain": plain_ms / batched_ms,
            "plain_loop_ms_by_order": {str(k): v[0] for k, v in plain_by_order.items()},
            "iterations_timed": reps, "frames": args.frames, "events_total": n_events,
            "rel_l2_batched_vs_plain_max": max(errs), "autotuned": list(best),
            "autotune_ms": {str(k): v for k, v in (timings or {}).items()},
            "generation_s": gen_s, "data": "synthetic (seeded per-frame phantoms)",
            "config": {"workload": "batched_96x96x48_64frames", "grid": grid,
                       "voxel_mm": wl0.voxel, "kernel_width": round(wl0.kernel_width, 4),
                       "tof_res_ps": wl0.tof_res_ps, "subsets": S_sub}}
    emit(line)
    return 0


def _pick(d, *keys):
    out = {}
    for k in keys:
        v = d
        for part in k.split("."):
            v = v.get(part) if isinstance(v, dict) else None
        out[k.replace(".", "_")] = v
    return out


def run_other_configs():
    """The other benchmark workloads (Siddon 64^3, batched frames, the differentiable
    projector, the large axial FOV), each run in this process after the default step's
    measurement, summarised (their full lines come from ``--workload NAME``)."""
    global _COLLECT
    plan = [
        ("config1_siddon64", ["--workload", "siddon64"],
         ("metric", "value", "unit", "ms_per_step", "e2e.value", "osem_iteration_ms",
          "roofline.bound", "roofline.frac", "cpu_baseline.value", "clocks.sm_mhz")),
        ("config3_batched96", ["--workload", "batched96"],
         ("metric", "value", "unit", "plain_loop_ms", "speedup_vs_plain",
          "rel_l2_batched_vs_plain_max", "autotuned")),
        ("config4_autograd128", ["--workload", "autograd128"],
         ("metric", "value", "unit", "adjoint_identity_rel_err", "frames", "events_per_frame",
          "gradient_finite")),
        ("config5_large256", ["--workload", "large256", "--no-variants", "--cpu-seconds", "4"],
         ("metric", "value", "unit", "ms_per_step", "e2e.value", "roofline.bound",
          "roofline.frac", "effmap.ms", "effmap.lors", "effmap.generated_ms",
          "cpu_baseline.value")),
    ]
    out = {}
    for name, argv, keys in plan:
        _COLLECT = []
        try:
            main(argv + ["--no-configs"])
            out[name] = _pick(_COLLECT[-1], *keys) if _COLLECT else {"error": "no line"}
        except Exception as exc:  # one configuration failing does not hide the others
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
        finally:
            _COLLECT = None
            torch.cuda.empty_cache()
    return out


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched96":
        return run_batched(args)
    if args.workload == "siddon64":
        return run_siddon(args)
    if args.workload == "autograd128":
        return run_autograd(args)
    if args.workload == "large256_recon":
        return run_large_recon(args)

    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    from srf_b200 import Image, profiling
    from srf_b200 import preprocess as PP

    if args.tuning:
        from srf_b200 import tuning
        tuning.set_tuning(*[int(v) for v in args.tuning.split(",")])
    wl, events, img_np, tof_bin, tof_sigma2 = workload_inputs(args.events, rank, dev,
                                                              args.workload)
    n_events = events.shape[0]
    model = model_for(wl, tof_bin, tof_sigma2)
    groups = PP.recon_process(events, wl.tof_res_ps)
    groups_in = groups  # recon_process order: the CPU baseline samples the head of each group
    if args.order:
        groups = PP.order_by_direction(groups)
    data = PP.split_listmode(groups)
    image = Image(torch.as_tensor(img_np, device=dev), wl.center, wl.size)
    n_lors = sum(data[a].lors.shape[0] for a in "xyz")
    work = algorithmic_work(model, data, image)

    def step():
        bp = project_back(model, image, data, args.combined)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(bp.data)
        return bp

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if clocks:
        clocks.start()
    timer = profiling.KernelTimer()
    from srf_b200 import _lib
    launches0 = _lib.call_raw("srf_launch_count")
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("bench_timed")
    with timer:
        start.record()
        for _ in range(args.steps):
            step()
        end.record()
    torch.cuda.nvtx.range_pop()
    gpu_launches = _lib.call_raw("srf_launch_count") - launches0
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    clk = clocks.stop() if clocks else None
    kern = timer.summary()
    ms = max_over_ranks(ms, world)
    total_lors = n_lors * world * args.steps
    value = total_lors / (ms / 1e3)

    # ---------------------------------------------------------------- e2e (public API)
    e2e = None
    if args.e2e_steps > 0:
        host_events = events.cpu().pin_memory()
        bi = host_events.numel() * 4
        bo = int(np.prod(wl.grid)) * 4

        def compute(ev):
            g = PP.recon_process(ev, wl.tof_res_ps)
            if args.order:
                g = PP.order_by_direction(g)
            d = PP.split_listmode(g)
            bp = project_back(model, image, d, args.combined)
            if world > 1:
                import torch.distributed as dist
                dist.all_reduce(bp.data)
            return bp.data

        pipelined_e2e(host_events, compute, 1, dev)  # warm-up
        barrier(world)
        e_ms = max_over_ranks(pipelined_e2e(host_events, compute, args.e2e_steps, dev), world)
        e2e = {"value": n_events * world * args.e2e_steps / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
               "ms_per_step": e_ms / args.e2e_steps,
               "path": "pinned host events -> recon_process -> projection -> backprojection "
                       "-> pinned host image; step k+1's upload overlaps step k"}

    variants = None
    if args.variants:
        variants = time_variants(wl, data, image, tof_bin, tof_sigma2, args.combined, world)

    # ---------------------------------------------------------------- effmap pass
    effmap = osem = None
    if args.effmap:
        from srf_b200 import recon
        args_e = (list(wl.grid), wl.center, wl.size, wl.scanner.inner_radius,
                  wl.scanner.axial_length)
        recon.efficiency_map(model, effmap_source(args, wl, 16_000_000, 78, dev), *args_e,
                             order=args.order)  # warm-up: one full chunk
        src = effmap_source(args, wl, wl.n_effmap, 77, dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        effinv, _ = recon.efficiency_map(model, src, *args_e, order=args.order)
        e1.record()
        torch.cuda.synchronize()
        e_ms = max_over_ranks(e0.elapsed_time(e1), world)
        effmap = {"lors": wl.n_effmap, "ms": e_ms, "lors_per_s": wl.n_effmap / (e_ms / 1e3),
                  "chunk": src.chunk,
                  "source": args.effmap_source,
                  "path": ("random crystal pairs (SplitMix64) made inside the binning and map "
                           "kernels from each LOR's number, map_process per LOR, no LOR array "
                           "-> TOR maplors of each axis group -> crop, normalise, invert"
                           if args.effmap_source == "generated" else
                           "random crystal pairs generated on the device per chunk -> "
                           "map_process -> " + ("records ordered by direction -> "
                                                if args.order else "")
                           + "TOR maplors of each axis group -> crop, normalise, invert")}
        if args.effmap_source == "tensor":
            # the same pass with LORs made inside the map kernels (no LOR array)
            gen = argparse.Namespace(**{**vars(args), "effmap_source": "generated"})
            recon.efficiency_map(model, effmap_source(gen, wl, 16_000_000, 78, dev), *args_e)
            torch.cuda.synchronize()
            e0.record()
            recon.efficiency_map(model, effmap_source(gen, wl, wl.n_effmap, 77, dev), *args_e)
            e1.record()
            torch.cuda.synchronize()
            effmap["generated_ms"] = max_over_ranks(e0.elapsed_time(e1), world)
        if wl.name == "tor_tof_128x128x64_10M" and world == 1:
            osem = time_osem(model, data, effinv, wl, dev)

    # ---------------------------------------------------------------- roofline
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    useful = sum(w["useful"] for w in work.values())
    slots = sum(w["slots"] for w in work.values())
    n_groups = sum(1 for w in work.values() if w["lors"] > 0)
    image_bytes = int(np.prod(wl.grid)) * 4
    roof = roofline(kern, args.steps, n_lors, n_groups, useful, slots, image_bytes, hbm_peak,
                    peak_src, wl.name)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            gh = {a: groups_in[a].cpu().numpy() for a in "xyz"}
            base = cpu_baseline(gh, wl, tof_bin, tof_sigma2, img_np, args.cpu_seconds)
        except Exception as exc:  # reported, never fatal for the GPU number
            base = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                    "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {"metric": METRICS[args.workload], "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded events from a cylinder phantom)",
                "config": {"workload": wl.name, "grid": list(wl.grid), "voxel_mm": wl.voxel,
                           "events_per_rank": int(n_events), "lors_per_rank": int(n_lors),
                           "kernel_width": round(wl.kernel_width, 4), "tof_res_ps": wl.tof_res_ps,
                           "tof_bin_mm": tof_bin, "tof_sigma2": tof_sigma2,
                           "groups": {a: w["lors"] for a, w in work.items()},
                           "parallelism": f"events sharded, {world} rank(s)",
                           "l2": "inputs larger than L2 (%d MB LOR records per rank)"
                                 % (n_lors * 40 // 10**6),
                           "tuning": args.tuning or "automatic"},
                "roofline": roof, "cpu_baseline": base, "e2e": e2e,
                "gpu_launches": gpu_launches, "clocks": clk, "variants": variants,
                "effmap": effmap, "osem": osem}
        if args.configs and world == 1 and args.workload == "tor128":
            line["configs"] = run_other_configs()
        emit(line)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
