"""Benchmark of the per-edit SVDAG editing path on B200 (one JSON line on rank 0).

Step = one edit of the seeded C0 stream (sphere add/remove near the surface of a depth-10 fBm
terrain, radius U{4..64}) followed by one 256x256 primary-ray frame (edit-to-visible).
value = edited voxels per second over the timed steps (Mvox/s), with p50/p99 edit-to-visible
latency beside it; `e2e` repeats the steps through the C ABI with the edit read from host memory
and the hit buffer copied back to pinned host memory every step. The slab-hash find/insert kernels
are measured on the 2^24-key microbenchmark and give the `roofline` object.

--impl reference times the reference algorithm on the host cores (the CPU oracle restatement of the
MyGpuDag pipeline; the reference has no CPU implementation of that pipeline) on the same config.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu-svdag-editing_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

LEVELS = 10
TERRAIN = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70)
EDIT_SEED = 2024
FRAME = 256
METRIC = "p99 edit latency & edited Mvox/s, served vs per-edit, bit-exact DAG, 1 B200"
HBM_FALLBACK_GBS = 6650.0


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def c0_edits(n, seed=EDIT_SEED):
    """Sphere edits of config 0: centre within +-32 voxels of the surface, radius U{4..64},
    50% add / 50% remove, add material U[0,8). Heights come from the terrain definition."""
    from oracle import oracle  # the terrain height function is shared with the checker

    L = oracle.lib()
    p = oracle.TerrainParams(**TERRAIN)
    rng = np.random.default_rng(seed)
    g = 1 << LEVELS
    out = []
    for _ in range(n):
        x, z = (int(v) for v in rng.integers(0, g, 2))
        h = L.oracle_terrain_height(p, LEVELS, x, z)
        c = (float(x + rng.integers(-32, 33)), float(h + rng.integers(-32, 33)), float(z + rng.integers(-32, 33)))
        r = float(rng.integers(4, 65))
        add = bool(rng.integers(0, 2))
        out.append((0 if add else 1, int(rng.integers(0, 8)), c, r))
    return out


class ClockSampler:
    """SM clock and clock-event reasons polled through NVML every 5 ms during the timed region
    (the per-edit steps are far shorter than nvidia-smi's 200 ms sampling period)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, cuda_device: int):
        self.cuda_device = cuda_device
        self.samples = []
        self.max_mhz = None
        self.handle = None
        self._stop = None

    def _open(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.cuda_device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0".upper()
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(0)
        self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        return pynvml

    def __enter__(self):
        import threading

        try:
            nv = self._open()
        except Exception:
            return self
        self._stop = threading.Event()

        def loop():
            while not self._stop.is_set():
                try:
                    mhz = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
                    try:
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                    except Exception:
                        rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.handle)
                    self.samples.append((mhz, rs))
                except Exception:
                    pass
                self._stop.wait(0.005)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *a):
        if self._stop is not None:
            self._stop.set()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        mhz = [m for m, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples), "source": "nvml, 5 ms"}


# ------------------------------------------------------------------ C1 hash microbenchmark

def c1_keys(n_unique, seed=1):
    """DAG-node keys: child-mask byte of popcount U{1..8}, then that many pointers U[0, 2^28)."""
    rng = np.random.default_rng(seed)
    pc = rng.integers(1, 9, n_unique)
    perm = np.argsort(rng.random((n_unique, 8)), axis=1)
    bits = (np.arange(8)[None, :] < pc[:, None])
    masks = np.zeros(n_unique, dtype=np.uint32)
    for j in range(8):
        masks |= np.where(bits[:, j], np.uint32(1) << perm[:, j].astype(np.uint32), 0).astype(np.uint32)
    sizes = (1 + pc).astype(np.int64)
    offs = np.zeros(n_unique, dtype=np.int64)
    offs[1:] = np.cumsum(sizes)[:-1]
    words = rng.integers(0, 1 << 28, int(sizes.sum()), dtype=np.uint32)
    words[offs] = masks
    return words, offs, sizes


def gather_keys(words, offs, sizes, order):
    s = sizes[order]
    o = np.zeros(len(order), dtype=np.int64)
    o[1:] = np.cumsum(s)[:-1]
    idx = np.repeat(offs[order] - o, s) + np.arange(int(s.sum()))
    return words[idx], o.astype(np.uint32), s


def run_hash_bench(svdag, torch, stream, n_total=1 << 24, load_factor=20, lanes=8, reps=3, pool=6 << 30):
    """Insert 2^24 keys (50% duplicates, stored twice as the reference's add does), then 2^24 finds
    (50% hits). Algorithmic bytes (per key of k words): find 4k + 32 + 4k*hit + 4, insert 4k + 32 + 4k + 4."""
    n_unique = n_total // 2
    words, offs, sizes = c1_keys(n_unique)
    rng = np.random.default_rng(3)
    ins_order = rng.permutation(np.concatenate([np.arange(n_unique), np.arange(n_unique)]))
    iw, io, isz = gather_keys(words, offs, sizes, ins_order)
    fw2, fo2, fs2 = c1_keys(n_unique, seed=2)  # fresh keys (misses)
    hit_sel = rng.permutation(n_unique)
    hw, ho, hs = gather_keys(words, offs, sizes, hit_sel)
    fw = np.concatenate([hw, fw2])
    fo = np.concatenate([ho, fo2.astype(np.uint32) + np.uint32(len(hw))])
    fsz = np.concatenate([hs, fs2])
    perm = rng.permutation(n_total)
    fw, fo, fsz = gather_keys(fw, fo.astype(np.int64), fsz, perm)
    is_hit = np.concatenate([np.ones(n_unique, bool), np.zeros(n_unique, bool)])[perm]

    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).astype(np.uint32).view(np.int32)).cuda()
    d_iw, d_io, d_fw, d_fo = dev(iw), dev(io), dev(fw), dev(fo)
    out = torch.empty(n_total, dtype=torch.int32, device="cuda")
    # buckets per size class ~ items of that class / load factor (stored items = 2^24)
    cls_items = np.bincount(isz - 2, minlength=9)[:9]
    buckets = np.maximum(1, cls_items // load_factor + 1).astype(np.uint32)
    ins_bytes = float(np.sum(4 * isz + 32 + 4 * isz + 4))
    find_bytes = float(np.sum(4 * fsz + 32 + 4 * fsz * is_hit + 4))
    res = {"insert_ms": [], "find_ms": []}
    for r in range(reps):
        dag = svdag.MyGPUHashDAG(10, pool_bytes=pool, scratch_bytes=min(1 << 30, pool // 4))
        tbl = dag.create_table(0, buckets)
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        with torch.cuda.stream(stream):
            e0.record(stream)
            tbl.add(d_iw, d_io, n_total, len(iw), out, lanes=lanes, stream=stream)
            e1.record(stream)
            tbl.find(d_fw, d_fo, n_total, len(fw), out, lanes=lanes, stream=stream)
            e2.record(stream)
        stream.synchronize()
        dag.sync()
        res["insert_ms"].append(e0.elapsed_time(e1))
        res["find_ms"].append(e1.elapsed_time(e2))
        if r == reps - 1:
            found = out.cpu().numpy().view(np.uint32) != 0xFFFFFFFF
            res["find_hit_rate"] = float(found.mean())
            res["hits_correct"] = bool(np.all(found[is_hit]))
            st = tbl.stats()
            res["stored_items"] = int(st.items)
            res["overflow_slabs"] = int(st.overflow_slabs)
        del tbl
        dag.free()
    ins = min(res["insert_ms"]) / 1e3
    fnd = min(res["find_ms"]) / 1e3
    return {
        "keys": n_total, "load_factor": load_factor, "lanes": lanes,
        "insert_ms": ins * 1e3, "find_ms": fnd * 1e3,
        "insert_mkeys_s": n_total / ins / 1e6, "find_mkeys_s": n_total / fnd / 1e6,
        "insert_gbs": ins_bytes / ins / 1e9, "find_gbs": find_bytes / fnd / 1e9,
        "find_bytes_per_launch": find_bytes, "insert_bytes_per_launch": ins_bytes,
        **{k: v for k, v in res.items() if not k.endswith("_ms")},
    }


# ------------------------------------------------------------------ per-edit path

def run_mine(args):
    import torch

    import svdag

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream()
    n_edits = args.warmup + args.steps
    edits = c0_edits(max(n_edits, 64))
    dag = svdag.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30)
    dag.build_terrain(**TERRAIN, stream=stream)
    params = svdag.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), FRAME, FRAME)
    hits = torch.empty(FRAME * FRAME * 68, dtype=torch.uint8, device="cuda")
    host_hits = torch.empty(FRAME * FRAME * 68, dtype=torch.uint8, pin_memory=True)

    def mk(i):
        tool, mat, c, r = edits[i % len(edits)]
        e = svdag.Edit(tool=tool, material=mat)
        e.center[:] = list(c)
        e.radius = r
        return e

    # warm-up (also collects per-edit edited-voxel counts of the whole stream on a scratch replay)
    for i in range(args.warmup):
        dag.edit(mk(i), stream=stream)
        dag.trace(params, hits, stream=stream)
    stream.synchronize()
    dag.sync(stream)

    # device-resident timed region: K edits + K frames
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    edited = 0
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        t_start.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            dag.edit(mk(args.warmup + k), stream=stream)
            dag.trace(params, hits, stream=stream)
            ev[k][1].record(stream)
            edited += dag.last_edit_stats(stream).edited_voxels  # host read of the step's counters
        t_end.record(stream)
        torch.cuda.synchronize()
    total_ms = t_start.elapsed_time(t_end)
    lat = sorted(a.elapsed_time(b) for a, b in ev)
    status = dag.last_edit_stats(stream).status

    # e2e: same steps through the C ABI with the edit from host memory and the hit buffer read back
    e2e_dag = svdag.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30)
    e2e_dag.build_terrain(**TERRAIN, stream=stream)
    for i in range(args.warmup):
        e2e_dag.edit(mk(i), stream=stream)
    stream.synchronize()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_edited = 0
    torch.cuda.synchronize()
    e_start.record(stream)
    for k in range(args.steps):
        e2e_dag.edit(mk(args.warmup + k), stream=stream)
        e2e_dag.trace(params, hits, stream=stream)
        with torch.cuda.stream(stream):
            host_hits.copy_(hits, non_blocking=True)
        e2e_edited += e2e_dag.last_edit_stats(stream).edited_voxels
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e_start.elapsed_time(e_end)

    # batched form: the same K edits (after the same warm-up) in one persistent launch
    b_dag = svdag.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30)
    b_dag.build_terrain(**TERRAIN, stream=stream)
    for i in range(args.warmup):
        b_dag.edit(mk(i), stream=stream)
    stream.synchronize()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record(stream)
    nrec = b_dag.edit_batch([mk(args.warmup + k) for k in range(args.steps)], stream=stream)
    b1.record(stream)
    torch.cuda.synchronize()
    b_ms = b0.elapsed_time(b1)
    b_edited = sum(r.edited_voxels for r in b_dag.edit_records(nrec, stream))
    b_dag.free()

    hash_res = run_hash_bench(svdag, torch, stream, lanes=args.hash_lanes, load_factor=args.hash_lf)
    t_max = total_ms
    if dist:
        t = torch.tensor([total_ms, e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max, e2e_ms = float(t[0]), float(t[1])
        cnt = torch.tensor([float(edited), float(e2e_edited)], device="cuda", dtype=torch.float64)
        dist.all_reduce(cnt)
        edited, e2e_edited = cnt[0].item(), cnt[1].item()
    peak, peak_kind = measured_peak_gbs()
    find_gbs = hash_res["find_gbs"]
    line = {
        "metric": METRIC,
        "value": edited / (t_max / 1e3) / 1e6,
        "unit": "edited Mvox/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded procedural fBm terrain and seeded edit stream)",
        "config": {"workload": "c0 per-edit: depth-10 (1024^3) fBm terrain, sphere add/remove r U{4..64} "
                               "near the surface, 256x256 primary-ray frame after each edit",
                   "levels": LEVELS, "frame": [FRAME, FRAME], "parallelism": f"replicas x{world}",
                   "l2": "DAG and tables resident; steps edit different regions"},
        "p50_edit_to_visible_ms": lat[len(lat) // 2],
        "p99_edit_to_visible_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
        "edit_status": int(status),
        "e2e": {"value": e2e_edited / (e2e_ms / 1e3) / 1e6, "unit": "edited Mvox/s",
                "h2d_bytes_per_step": 56, "d2h_bytes_per_step": FRAME * FRAME * 68 + 264},
        "roofline": {"bound": "hbm", "kernel": f"slab-hash find (C1, 2^24 keys, {args.hash_lanes} lane(s)/key)",
                     "achieved": find_gbs, "peak": peak, "unit": "GB/s", "frac": find_gbs / peak,
                     "peak_source": peak_kind, "traffic": None},
        "batched": {"edits": args.steps, "ms": b_ms, "ms_per_edit": b_ms / args.steps,
                    "edited_mvox_s": b_edited / (b_ms / 1e3) / 1e6, "note": "edits only, one persistent launch"},
        "hash_c1": hash_res,
        "clocks": clocks.summary(),
        "gpu_launches": args.steps * (4 * (LEVELS - 2) + 6),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line))
    dag.free()
    e2e_dag.free()
    if dist:
        dist.destroy_process_group()


def cpu_baseline(args, sample_edits=64):
    """The oracle restatement of the MyGpuDag pipeline on one host core, on the same C0 stream."""
    from oracle import oracle

    d = oracle.OracleDag(LEVELS)
    d.build_terrain(oracle.TerrainParams(**TERRAIN))
    edits = c0_edits(max(args.warmup + args.steps, 64))
    edited = 0
    t0 = time.perf_counter()
    for i in range(sample_edits):
        tool, mat, c, r = edits[i]
        e = oracle.Edit(tool=tool, material=mat)
        e.center[:] = list(c)
        e.radius = r
        edited += d.edit(e).edited_voxels
    dt = time.perf_counter() - t0
    return {"value": edited / dt / 1e6, "unit": "edited Mvox/s", "cores": 1, "kind": "port",
            "sample": f"first {sample_edits} edits of the C0 stream on the depth-10 terrain (edits only, no frames)"}


def run_reference(args):
    """Reference arm: the CPU restatement of the reference path (the reference's MyGpuDag pipeline has
    no CPU implementation) timed on the host, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle

    d = oracle.OracleDag(LEVELS)
    d.build_terrain(oracle.TerrainParams(**TERRAIN))
    edits = c0_edits(max(args.warmup + args.steps, 64))
    params = oracle.camera_params([512.0, 900.0, 512.0], [512.0, 512.0, 512.0], 60.0, FRAME, FRAME)
    threads = os.cpu_count() or 1

    def step(i):
        tool, mat, c, r = edits[i % len(edits)]
        e = oracle.Edit(tool=tool, material=mat)
        e.center[:] = list(c)
        e.radius = r
        st = d.edit(e)
        d.trace(params, threads=threads)
        return st.edited_voxels

    for i in range(args.warmup):
        step(i)
    lat, edited = [], 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        s = time.perf_counter()
        edited += step(args.warmup + k)
        lat.append((time.perf_counter() - s) * 1e3)
    dt = time.perf_counter() - t0
    lat.sort()
    v = edited / dt / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "edited Mvox/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded procedural fBm terrain and seeded edit stream)",
        "config": {"workload": "c0 per-edit: depth-10 (1024^3) fBm terrain, sphere add/remove r U{4..64} "
                               "near the surface, 256x256 primary-ray frame after each edit", "levels": LEVELS},
        "p50_edit_to_visible_ms": lat[len(lat) // 2], "p99_edit_to_visible_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
        "cpu_baseline": {"value": v, "unit": "edited Mvox/s", "cores": threads, "kind": "port",
                         "sample": "the timed steps themselves (edit single-threaded, frame on all cores)"},
        "e2e": {"value": v, "unit": "edited Mvox/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_mode_hash(args):
    """Only the C1 slab-hash microbenchmark (profiling entry point)."""
    import torch

    import svdag

    r = run_hash_bench(svdag, torch, torch.cuda.Stream(), n_total=args.hash_keys, lanes=args.hash_lanes,
                       load_factor=args.hash_lf, reps=args.hash_reps, pool=args.hash_pool)
    print(json.dumps({k: v for k, v in r.items()}))


def run_mode_edit(args):
    """Only the per-edit path: depth-10 terrain, warm-up edits, then K edits each followed by a frame
    (profiling entry point)."""
    import torch

    import svdag

    edits = c0_edits(max(args.warmup + args.steps, 64))
    dag = svdag.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30)
    dag.build_terrain(**TERRAIN)
    params = svdag.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), FRAME, FRAME)
    hits = torch.empty(FRAME * FRAME * 68, dtype=torch.uint8, device="cuda")
    te, tt, phases = [], [], []
    for i in range(args.warmup + args.steps):
        tool, mat, c, r = edits[i % len(edits)]
        e = svdag.Edit(tool=tool, material=mat)
        e.center[:] = list(c)
        e.radius = r
        a, b, d = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        dag.edit(e)
        b.record()
        dag.trace(params, hits)
        d.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            te.append(a.elapsed_time(b))
            tt.append(b.elapsed_time(d))
            pt = dag.last_edit_phase_times()
            phases.append([round(float(x - pt[0]) / 1e3, 2) for x in pt])
    dag.sync()
    print(json.dumps({"edit_ms_median": statistics.median(te), "trace_ms_median": statistics.median(tt),
                      "edit_ms": te, "trace_ms": tt, "phase_us": phases[:4]}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--mode", default="full", choices=["full", "hash", "edit"],
                    help="full = the benchmark line; hash / edit run one sub-workload (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--hash-keys", type=int, default=1 << 24)
    ap.add_argument("--hash-lanes", type=int, default=1)
    ap.add_argument("--hash-lf", type=int, default=20)
    ap.add_argument("--hash-reps", type=int, default=3)
    ap.add_argument("--hash-pool", type=int, default=6 << 30)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "hash":
        run_mode_hash(args)
    elif args.mode == "edit":
        run_mode_edit(args)
    else:
        run_mine(args)


if __name__ == "__main__":
    main()
