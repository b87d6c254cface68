"""Benchmark of the SVDAG editing path on B200 (one JSON line on rank 0).

Default workload (--mode serve): the served edit stream on the at-scale scene. The scene is the
depth-17 (131072^3) fBm terrain with 8 octaves and 4096 boxes/spheres on the surface, built on the
GPU; the stream is Poisson edit arrivals (add / remove / paint / copy 35/35/20/10, radius
log-uniform 2..2048, centres on the surface) with 1920x1080 frame requests at 60 Hz, undo history 32
deep, admission under a 120 GB cap. The same timed request stream is replayed against the serving
form (continuous batching) and against the plain per-edit path (one request at a time, an edit then a
frame); `value` is the served p99 edit-to-visible latency, with the plain path's beside it.
`e2e` repeats the served replay with every frame copied to pinned host memory.

A step is one window of `--window` seconds of the stream; W windows are replayed untimed first, then
K windows in one continuous replay. Other modes (profiling entry points): c0 (depth-10 per-edit
path), c2 (the at-scale edit sequence), c3 (256 uneven edits, batched vs plain), hash (the 2^24-key
slab-hash microbenchmark), hashmap (the reference's table benchmark over every slab layout).

--impl reference times the reference algorithm on the host cores: the CPU restatement of the
MyGpuDag pipeline (the reference has no CPU implementation of it) on a bounded sample of the same
stream, each edit on the scene clipped to its footprint.
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

METRIC = "p99 edit latency & edited Mvox/s, served vs per-edit, bit-exact DAG, 1 B200"
HBM_FALLBACK_GBS = 6650.0
POOL_CAP = 120 << 30
C0_FRAME = 256


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class profiled:
    """Marks the measured region for a profiler started with --profile-from-start off (cudaProfilerStart /
    cudaProfilerStop; no effect otherwise), so that scene construction is left out of captures."""

    def __enter__(self):
        import torch

        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        return self

    def __exit__(self, *a):
        import torch

        torch.cuda.synchronize()
        torch.cuda.profiler.stop()


def pct(a, q):
    return float(np.percentile(np.asarray(a, dtype=np.float64), q)) if len(a) else None


class ClockSampler:
    """SM clock and clock-event reasons polled through NVML every 5 ms during the timed region."""

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


def run_hash_bench(svdag, torch, stream, n_total=1 << 24, load_factor=16, lanes=1, reps=3, pool=6 << 30):
    """Insert 2^24 keys (50% duplicates, stored twice as the reference's add does), then 2^24 finds
    (50% hits). 16 stored items per bucket gives the configuration's 2^20 buckets. Algorithmic bytes (per key of k words): find 4k + 32 + 4k*hit + 4, insert 4k + 32 + 4k + 4."""
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


# ------------------------------------------------------------------ the served stream (C4 on the C2 scene)

def c2_camera(svdag, levels, width=1920, height=1080):
    g = float(1 << levels)
    return svdag.get_trace_params((0.5 * g - 6000.0 * g / 131072, 0.62 * g, 0.5 * g - 6000.0 * g / 131072),
                                  (0.5 * g, 0.52 * g, 0.5 * g), width, height)


def make_scene(svdag, w, levels, phase_kernels=False, pool_gb=0.0, persistent=False):
    # 86 GiB at depth 17 (the 64 GiB item region the 32-bit handle reaches, its slab headers and a
    # 16 GiB scratch arena); smaller scenes get a share of it by surface area (4^(levels-17)), at
    # least 2 GiB
    shrink = 4 ** max(0, w.C2_LEVELS - levels)
    pool = int(pool_gb * (1 << 30)) if pool_gb else max(2 << 30, min(POOL_CAP, 86 << 30) // shrink)
    dag = svdag.MyGPUHashDAG(levels, pool_bytes=pool, scratch_bytes=max(512 << 20, (16 << 30) // shrink),
                             undo_depth=32, phase_kernels=phase_kernels, persistent=persistent)
    terrain = make_terrain(w, levels)
    dag.build_terrain(**terrain)
    dag.sync()
    return dag, terrain


def max_over_ranks(values, dist=None, device="cuda"):
    """Element-wise max of floats over all ranks: a replica job's latency is its slowest rank's."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def summarize(res, n_edits, duration_s=None, edits=None):
    """Latency (ms) and throughput of a replay; res = edits then frames. `sustained`: the last edit
    became visible within 10 % (+0.25 s) of the end of the stream, so no backlog built up. With the
    edits given, the p99 per radius band too."""
    ed = res[:n_edits]
    lat = (ed["visible_s"] - ed["submit_s"]) * 1e3
    fr = res[n_edits:]
    flat = (fr["visible_s"] - fr["submit_s"]) * 1e3
    span = float(res["visible_s"].max() - res["submit_s"].min()) if len(res) else 0.0
    vox = float(ed["edited_voxels"].sum())
    launches = len(set(res["launch"].tolist()))
    out = {"edits": int(n_edits), "ok": int((ed["status"] == 0).sum()), "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
           "max_ms": float(lat.max()) if len(lat) else None, "frame_p99_ms": pct(flat, 99),
           "edited_mvox_s": vox / span / 1e6 if span > 0 else None, "launches": launches,
           "mean_edits_per_launch": float(n_edits) / max(1, len(set(ed["launch"].tolist()))), "span_s": span}
    if duration_s is not None:
        out["sustained"] = bool(span <= 1.1 * duration_s + 0.25)
    if edits is not None and len(edits) == n_edits:
        radius = np.array([e.radius for e in edits])
        out["p99_ms_by_radius"] = {f"{lo:g}-{hi:g}": pct(lat[(radius >= lo) & (radius < hi)], 99)
                                   for lo, hi in ((0, 64), (64, 512), (512, 1e9)) if ((radius >= lo) & (radius < hi)).any()}
    return out


def require_ok(res, n_edits, what, memory=None):
    """Every edit of a replay must have succeeded: a latency over failed edits measures nothing."""
    st = res["status"][:n_edits]
    bad = np.nonzero(st != 0)[0]
    if len(bad):
        i = int(bad[0])
        raise SystemExit(f"bench: {what}: {len(bad)} of {n_edits} edits failed; first: edit {i} with status "
                         f"{int(st[i])} (launch {int(res['launch'][i])}); server memory: {memory}")


def replay(svdag, dag, cam, edits, times, frames, plain=False, copy_frames=False, counters=None, memory=None):
    """Serves a timed stream; `counters` and `memory` (dicts) receive the server's frame counters and
    memory accounting (in-loop collections)."""
    with svdag.Server(dag, cam, max_batch=256, max_inflight=2, memory_cap_bytes=POOL_CAP, plain=plain,
                      copy_frames=copy_frames) as srv:
        res = srv.replay(edits, times, frames)
        if counters is not None:
            counters.update(srv.counters())
        if memory is not None:
            memory.update(srv.memory())
        return res


def edit_algorithmic_bytes(records):
    """Per edit: every intermediate SVO item written by the top-down phases and read by the bottom-up
    ones (44 + 44 bytes with its representative and handle), one table find per distinct item (a
    32-byte slab header and a 40-byte candidate), 40 bytes per inserted item."""
    return float(sum(r.svo_items * 88 + r.unique_items * 72 + r.new_items * 40 for r in records))


def stream_of(w, levels, rate, duration, seed, height=None):
    rmax = 2048.0 * (1 << levels) / 131072
    return w.c4_stream(rate, duration, seed=seed, levels=levels, rmax=rmax, terrain=make_terrain(w, levels),
                       copy_offset=int(1024 * (1 << levels) / 131072), height=height)


def trace_rays_s(svdag, torch, dag, cam, frames=10):
    """Whole 1920x1080 frames of the scene (CUDA events on the tracer's stream)."""
    tracer = svdag.DAGTracer(cam.width, cam.height)
    stream = torch.cuda.Stream()
    for _ in range(3):
        tracer.resolve_paths(cam, dag, stream=stream.cuda_stream)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
    torch.cuda.synchronize()
    for a, b in ev:
        a.record(stream)
        tracer.resolve_paths(cam, dag, stream=stream.cuda_stream)
        b.record(stream)
    torch.cuda.synchronize()
    ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    hits = tracer.hits_numpy()
    return {"frame_ms": ms, "rays_s": cam.width * cam.height / (ms / 1e3),
            "hit_fraction": float((hits["material"] != 255).mean())}


def run_serve(args):
    import torch

    import svdag
    import svdag.workloads as w

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    levels = args.levels
    dur_w, dur_k = args.warmup * args.window, args.steps * args.window
    # warm-up and timed streams (different seeds, so the timed edits are new work)
    tw, ew, fw = stream_of(w, levels, args.rate, dur_w, 40 + rank)
    tk, ek, fk = stream_of(w, levels, args.rate, dur_k, 4 + rank)
    cam = c2_camera(svdag, levels)
    out = {}

    def prepared_scene(plain):
        """The scene built on the GPU, the launch form tuned on the first warm-up edits (applied for
        real), the rest of the warm-up stream served, then a collection (undo history kept)."""
        dag, _ = make_scene(svdag, w, levels, persistent=args.persistent)
        tuning = dag.autotune(edits=ew[:64])
        mem = {}
        res = replay(svdag, dag, cam, ew[64:], [t - tw[64] for t in tw[64:]] if len(ew) > 64 else [], fw, plain=plain,
                     memory=mem)
        require_ok(res, max(0, len(ew) - 64), f"{'plain' if plain else 'served'} warm-up", mem)
        dag.garbage_collect(keep_history=True)
        return dag, {"persistent_leaves": tuning.persistent_leaves, "graph_us_small": tuning.graph_us_small,
                     "persistent_us_small": tuning.persistent_us_small}

    # Each replay below runs on a scene of its own: a depth-17 DAG keeps growing with the detail the
    # edits add (undo history and garbage are collected, live data is not), and its 32 GiB item region
    # holds the warm-up, a timed stream and some more, not every stream of the run.
    for name, plain in (("served", False), ("plain", True)):
        dag, tuning = prepared_scene(plain)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        mem, frames = {}, {}
        with ClockSampler(local) as clocks, profiled():
            t0 = time.perf_counter()
            res = replay(svdag, dag, cam, ek, tk, fk, plain=plain, memory=mem, counters=frames)
            wall = time.perf_counter() - t0
        torch.cuda.synchronize()
        require_ok(res, len(ek), f"{name} timed stream", mem)
        out[name] = summarize(res, len(ek), dur_k, ek)
        out[name].update(wall_s=wall, memory=mem, frames=frames, tuning=tuning)
        if name == "served":
            out["clocks"] = clocks.summary()
            # the dominant kernel: one window of the stream as one batched launch
            dag.garbage_collect(keep_history=True)
            nwin = max(1, len(ek) // max(1, args.steps))
            batch = ek[:nwin]
            stream = torch.cuda.Stream()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            nrec = dag.edit_batch(batch, stream=stream.cuda_stream)
            b.record(stream)
            torch.cuda.synchronize()
            recs = dag.edit_records(nrec)
            bad = [i for i, r in enumerate(recs) if r.status != 0]
            if bad:
                raise SystemExit(f"bench: batched window: edit record {bad[0]} has status {recs[bad[0]].status}")
            out["batch"] = {"edits": len(batch), "ms": a.elapsed_time(b), "bytes": edit_algorithmic_bytes(recs),
                            "svo_items": int(sum(r.svo_items for r in recs))}
            out["used_gb"] = dag.stats().item_region_used_bytes / 1e9
            out["trace"] = trace_rays_s(svdag, torch, dag, cam)
        dag.free()
        del dag
    # e2e: the timed stream served again, on a fresh scene, with every frame copied to pinned host memory
    dag, _ = prepared_scene(False)
    frame_counters, mem = {}, {}
    res_e2e = replay(svdag, dag, cam, ek, tk, fk, copy_frames=True, counters=frame_counters, memory=mem)
    require_ok(res_e2e, len(ek), "e2e stream", mem)
    out["e2e"] = summarize(res_e2e, len(ek), dur_k)
    out["e2e"].update(frames=frame_counters, memory=mem)
    dag.free()
    del dag
    # offered-load sweep: the same stream shape at other rates, served then plain, each from a
    # collected region of one more fresh scene
    out["sweep"] = []
    sweep = [float(r) for r in args.sweep.split(",") if r]
    if sweep:
        dag, _ = prepared_scene(False)
        for i, rate in enumerate(sweep):
            dur = min(8.0, max(2.0, 400.0 / rate))
            ts, es, fs = stream_of(w, levels, rate, dur, 200 + 10 * i + rank)
            point = {"rate_edits_per_s": rate, "duration_s": dur}
            for name, plain in (("served", False), ("plain", True)):
                dag.garbage_collect(keep_history=True)
                mem = {}
                res = replay(svdag, dag, cam, es, ts, fs, plain=plain, memory=mem)
                require_ok(res, len(es), f"{name} at {rate:g} edits/s", mem)
                point[name] = summarize(res, len(es), dur)
                point[name]["gc_runs"] = mem.get("gc_runs")
            point["p99_served_over_plain"] = point["served"]["p99_ms"] / point["plain"]["p99_ms"]
            out["sweep"].append(point)
        dag.free()
        del dag
    # the batched form on scattered small edits (runs of them land in disjoint subtrees, built side by
    # side), against the per-edit path
    batching = None
    if not args.no_batching:
        small = w.c3_edits(levels=levels, terrain=make_terrain(w, levels), rmax=16.0, seed=5)
        batching = {"small_scattered_256": c3_compare(svdag, w, torch, levels, small)}
    peak, peak_kind = measured_peak_gbs()
    trace_c0 = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu_c0, cpu_hits = cpu_trace_c0()
        trace_c0 = {"gpu": gpu_trace_c0(svdag, torch, cpu_c0, cpu_hits, peak), "cpu": cpu_c0}
    hash_res = []
    if not args.no_hash:
        for lf in (16, 96):
            for lanes in (1, 32):
                hash_res.append(run_hash_bench(svdag, torch, torch.cuda.Stream(), lanes=lanes, load_factor=lf))
    p99 = out["served"]["p99_ms"]
    p99, out["plain"]["p99_ms"], out["e2e"]["p99_ms"] = max_over_ranks([p99, out["plain"]["p99_ms"], out["e2e"]["p99_ms"]], dist)
    bt = out["batch"]
    achieved = bt["bytes"] / (bt["ms"] / 1e3) / 1e9
    # frame bytes the server copied to host memory (incremental frames copy only their changed pixels)
    frame_d2h = out["e2e"]["frames"].get("frame_bytes_to_host", cam.width * cam.height * 68 * out["e2e"]["launches"])
    # the served/plain ratio at the highest offered load both paths sustain (the plain loop's p99 at a
    # load it cannot keep up with measures its queue, not its kernels)
    points = [(args.rate, out["served"], out["plain"])] + [(p["rate_edits_per_s"], p["served"], p["plain"]) for p in out["sweep"]]
    both = [pt for pt in points if pt[1]["sustained"] and pt[2]["sustained"]]
    head = max(both, key=lambda pt: pt[0]) if both else None
    fr = out["served"]["frames"]
    line = {
        "metric": METRIC,
        "value": p99,
        "unit": "ms (served p99 edit-to-visible)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": out["served"]["wall_s"] * 1e3 / args.steps,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded procedural scene and seeded Poisson request stream)",
        "config": {"workload": f"c4 served stream on the c2 scene: depth-{levels} fBm terrain (8 octaves) + "
                               f"{make_terrain(w, levels)['num_structures']} boxes/spheres, Poisson {args.rate:g} edits/s "
                               "add/remove/paint/copy 35/35/20/10, radius log-uniform 2..2048, 1920x1080 frames "
                               "at 60 Hz, undo depth 32, 120 GB cap",
                   "levels": levels, "rate_edits_per_s": args.rate, "window_s": args.window,
                   "frame": [cam.width, cam.height], "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (the DAG holds > 20 GB; edits land at random places)"},
        "served": out["served"], "plain": out["plain"],
        "p99_served_over_plain": p99 / out["plain"]["p99_ms"] if out["plain"]["p99_ms"] else None,
        "p99_served_over_plain_sustained": ({"rate_edits_per_s": head[0], "ratio": head[1]["p99_ms"] / head[2]["p99_ms"],
                                             "served_p99_ms": head[1]["p99_ms"], "plain_p99_ms": head[2]["p99_ms"]}
                                            if head else None),
        "sweep": out["sweep"],
        "edited_mvox_s_served": out["served"]["edited_mvox_s"],
        "e2e": {"value": out["e2e"]["p99_ms"], "unit": "ms (served p99 edit-to-visible, frames copied to host)",
                "h2d_bytes_per_step": int(56 * len(ek) / args.steps),
                "d2h_bytes_per_step": int((frame_d2h + 48 * len(ek)) / args.steps),
                "detail": out["e2e"]},
        "roofline": {"bound": "hbm", "kernel": "edit pipeline: one window of the stream as one batch (per-tool CUDA graphs of "
                               "the phase kernels, small edits in the persistent kernel or in subtree groups)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": None, "launch": bt},
        "trace_1080p": dict(out["trace"], bytes_per_ray_lower_bound=68 + 8 * levels,
                            hbm_frac_lower_bound=out["trace"]["rays_s"] * (68 + 8 * levels) / 1e9 / peak),
        "trace_c0": trace_c0,
        "batching": batching,
        "clocks": out["clocks"],
        # launch calls of the timed served replay: one per batch (a CUDA-graph replay or one persistent
        # kernel per run of small edits) and one per frame
        "gpu_launches": out["served"]["launches"] + fr.get("frames_whole", 0) + fr.get("frames_incremental", 0),
        "item_region_used_gb": out["used_gb"],
    }
    if hash_res:
        line["hash_c1"] = hash_res
        primary = hash_res[0]
        line["hash_roofline"] = {"kernel": f"slab-hash find (2^24 keys, load factor {primary['load_factor']}, "
                                           f"{primary['lanes']} lane(s)/key)",
                                 "achieved": primary["find_gbs"], "peak": peak, "unit": "GB/s",
                                 "frac": primary["find_gbs"] / peak,
                                 "insert_achieved": primary["insert_gbs"], "insert_frac": primary["insert_gbs"] / peak}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(args, levels)["cpu_baseline"]
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def make_terrain(w, levels):
    if levels == w.C2_LEVELS:
        return w.C2_TERRAIN
    return dict(w.C2_TERRAIN, num_structures=max(16, 4096 >> (2 * (w.C2_LEVELS - levels))))


# ------------------------------------------------------------------ CPU baseline / reference arm

def edit_box(e):
    """Voxel box the edit can read or change (copies: source and destination)."""
    c, r = np.array(e.center, dtype=np.float64), float(e.radius) + 2.0
    if e.tool in (5, 7):
        d = np.array(e.dst, dtype=np.float64) + c - np.array(e.src, dtype=np.float64)
        lo, hi = np.minimum(c, d) - r, np.maximum(c, d) + r
    else:
        lo, hi = c - r, c + r
    return [int(np.floor(v)) for v in lo], [int(np.ceil(v)) + 1 for v in hi]


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(args, levels, budget_s=25.0, min_edits=64, hard_s=90.0):
    """The oracle (the CPU restatement of the reference pipeline; the reference's MyGpuDag path has no
    CPU implementation) on the leading edits of the timed stream, one edit per host thread at a time
    on every host core, each edit on the scene clipped to its box (the result inside the box equals
    the full scene's: edits are local). Times the edit only; the region build is not timed. At least
    `min_edits` edits, more while `budget_s` lasts. Loads no CUDA library: the stream's surface heights
    come from the oracle's own terrain function."""
    import concurrent.futures as cf
    import threading

    import svdag.workloads as w
    from oracle import oracle

    L = oracle.lib()
    params = oracle.TerrainParams(**make_terrain(w, levels))
    height = lambda lv, x, z, terrain: L.oracle_terrain_height(params, lv, x, z)
    _, ek, _ = stream_of(w, levels, args.rate, args.steps * args.window, 4, height=height)
    threads = host_threads()
    lock = threading.Lock()
    state = {"next": 0}
    start = time.perf_counter()
    results = []

    def worker():
        while True:
            with lock:
                i = state["next"]
                el = time.perf_counter() - start
                if i >= len(ek) or (i >= min_edits and el > budget_s) or el > hard_s:
                    return
                state["next"] = i + 1
            e = ek[i]
            d = oracle.OracleDag(levels)
            lo, hi = edit_box(e)
            d.build_scene_region(params, lo, hi)
            oe = oracle.Edit(tool=e.tool, material=e.material, radius=e.radius, noise_seed=e.noise_seed,
                             noise_cell_log2=e.noise_cell_log2)
            oe.center[:], oe.src[:], oe.dst[:] = list(e.center), list(e.src), list(e.dst)
            t0 = time.perf_counter()
            st = d.edit(oe)
            ms = (time.perf_counter() - t0) * 1e3
            with lock:
                results.append((i, ms, st.edited_voxels, float(e.radius)))
            del d

    with cf.ThreadPoolExecutor(threads) as ex:
        for f in [ex.submit(worker) for _ in range(threads)]:
            f.result()
    wall = time.perf_counter() - start
    results.sort()
    lat = [r[1] for r in results]
    vox = sum(r[2] for r in results)
    radii = [r[3] for r in results]
    p99 = pct(lat, 99)
    return {"p99_ms": p99, "p50_ms": pct(lat, 50), "mean_ms": float(np.mean(lat)), "edits": len(lat),
            "edited_mvox_s": vox / (sum(lat) / 1e3) / 1e6, "threads": threads,
            "cpu_baseline": {"value": p99, "unit": "ms (p99 edit latency, edit only)", "cores": threads, "kind": "port",
                             "sample": f"first {len(lat)} edits of the timed stream (radius {min(radii):.0f}..{max(radii):.0f}), "
                                       f"one edit per thread on {threads} host threads, each on the scene clipped to its "
                                       "box; edit time only, no frame, no queueing",
                             "p50_ms": pct(lat, 50), "edits_per_s_all_threads": len(lat) / wall,
                             "edited_mvox_s_all_threads": vox / wall / 1e6}}


def c0_trace_params(svdag):
    """The C0 frame: 256x256 primary rays of the depth-10 terrain from (512, 900, 512) towards the
    grid centre (get_trace_params is host Python: no CUDA library is loaded)."""
    return svdag.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), C0_FRAME, C0_FRAME)


def cpu_trace_c0(reps=3):
    """The oracle's tracer (a restatement of tracer.cu; the reference has no CPU tracer) on the C0
    frame, row bands on every host thread. Returns rays/s, the hit buffer and the visit counts the
    algorithmic bytes of the trace roofline come from."""
    import svdag
    import svdag.workloads as w
    from oracle import oracle

    threads = host_threads()
    o = oracle.OracleDag(w.C0_LEVELS)
    o.build_terrain(oracle.TerrainParams(**w.C0_TERRAIN))
    p = c0_trace_params(svdag)
    po = oracle.TraceParams()
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, f)[:] = list(getattr(p, f))
    po.width, po.height = p.width, p.height
    best, hits = None, None
    for _ in range(reps):
        t0 = time.perf_counter()
        hits = o.trace(po, threads)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    nodes, leaves, nhits = o.trace_counts(po)
    return {"rays_s": p.width * p.height / best, "threads": threads, "frame_ms": best * 1e3,
            "node_visits": nodes, "leaf_visits": leaves, "hits": nhits}, hits


def gpu_trace_c0(svdag, torch, cpu, cpu_hits, peak, frames=50):
    """The same C0 frame on the GPU (CUDA events over `frames` launches on the tracer's stream),
    checked pixel for pixel against the oracle's hit buffer. Algorithmic bytes per frame: 8 per node
    visit (header + child pointer), 12 per leaf visit, 68 per hit record written."""
    import svdag.workloads as w

    dag = svdag.MyGPUHashDAG(w.C0_LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30)
    dag.build_terrain(**w.C0_TERRAIN)
    p = c0_trace_params(svdag)
    tracer = svdag.DAGTracer(p.width, p.height)
    stream = torch.cuda.Stream()
    for _ in range(3):
        tracer.resolve_paths(p, dag, stream=stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(frames):
        tracer.resolve_paths(p, dag, stream=stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / frames
    hits = tracer.hits_numpy()
    exact = bool(np.array_equal(hits["path"], cpu_hits["path"]) and np.array_equal(hits["material"], cpu_hits["material"]))
    dag.free()
    rays = p.width * p.height
    alg = 8.0 * cpu["node_visits"] + 12.0 * cpu["leaf_visits"] + 68.0 * rays
    return {"rays_s": rays / (ms / 1e3), "frame_us": ms * 1e3, "bit_exact_vs_oracle": exact,
            "bytes_per_frame": alg, "hbm_frac": alg / (ms / 1e3) / 1e9 / peak}


def run_reference(args):
    """Reference arm: the CPU restatement of the reference path timed on the host cores, rank 0 only.
    No CUDA library is loaded (libsvdag.so stays unmapped)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    r = cpu_sample(args, args.levels)
    cb = r["cpu_baseline"]
    trace, _ = cpu_trace_c0()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": r["p99_ms"], "unit": "ms (p99 edit latency, edit only)",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["mean_ms"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded procedural scene and seeded request stream)",
        "config": {"workload": f"c4 stream edits on the c2 scene (depth {args.levels}), one edit per host thread on the CPU",
                   "levels": args.levels, "rate_edits_per_s": args.rate},
        "p50_ms": r["p50_ms"], "edits": r["edits"], "edited_mvox_s": r["edited_mvox_s"],
        "cpu_baseline": cb,
        "trace_c0_cpu": trace,
        "e2e": {"value": r["p99_ms"], "unit": "ms (p99 edit latency, edit only)", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


# ------------------------------------------------------------------ profiling entry points

def run_mode_hash(args):
    """Only the 2^24-key slab-hash microbenchmark."""
    import torch

    import svdag

    r = run_hash_bench(svdag, torch, torch.cuda.Stream(), n_total=args.hash_keys, lanes=args.hash_lanes,
                       load_factor=args.hash_lf, reps=args.hash_reps, pool=args.hash_pool)
    print(json.dumps(r))


def run_mode_hashmap(args):
    """The reference's table benchmark (extras/hashmap_bench/src/main.cu:560-720, defaults :850-873)
    over every slab layout: items of 2 words, a bulk add of 8M items, 1M finds at hit rates
    0/25/50/75/100 %, a second bulk add of 1M items, 64 items per bucket, room reserved for twice the
    items. Layouts: ticket_board, atomic64, acceleration, individual_chaining (svdag_alt_table_*) and
    compact (the level tables' layout; its keys are 2-word node keys, a one-bit child mask then a
    word). Each runs thread per key (lanes 1) and warp-hybrid / 32 lanes per key (lanes 32), except
    individual_chaining, which has only the thread-per-key form. Every phase is checked: all adds
    stored, exactly the expected finds hit."""
    import torch

    import svdag

    k = 2
    n0, n1, ns = args.hashmap_initial, args.hashmap_insert, args.hashmap_search
    rng = np.random.default_rng(11)
    keys = rng.integers(0, 1 << 32, (n0 + n1 + ns, k), dtype=np.uint64).astype(np.uint32)
    keys[:, 0] = (keys[:, 0] & 0xFFFFFF00) | (np.uint32(1) << (keys[:, 0] & 7))  # valid 2-word node keys
    init, more, never = keys[:n0], keys[n0:n0 + n1], keys[n0 + n1:]
    buckets = (n0 + n1) // 64 + 1
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).reshape(-1).view(np.int32)).cuda()
    d_init, d_more = d(init), d(more)
    searches = {}
    for pct in (0, 25, 50, 75, 100):
        hits = ns * pct // 100
        searches[pct] = (d(np.concatenate([init[rng.permutation(n0)[:hits]], never[:ns - hits]])), hits)
    offs = {n: torch.arange(0, k * n, k, dtype=torch.int32, device="cuda") for n in {n0, n1, ns}}
    stream = torch.cuda.Stream()
    peak, peak_kind = measured_peak_gbs()
    dag = svdag.MyGPUHashDAG(6, pool_bytes=max(1 << 30, 64 * (n0 + n1) * 4), scratch_bytes=64 << 20)
    results = []
    for layout in ("ticket_board", "atomic64", "acceleration", "individual_chaining", "compact"):
        for lanes in ((1,) if layout == "individual_chaining" else (1, 32)):
            if layout == "compact":
                per_size = np.zeros(svdag.NUM_SIZE_CLASSES, np.uint32)
                per_size[0] = buckets
                tbl = dag.create_table(svdag.KIND_NODE, per_size)
                add = lambda kd, n, out: tbl.add(kd, offs[n], n, k * n, out, lanes=lanes, stream=stream)
                find = lambda kd, n, out: tbl.find(kd, offs[n], n, k * n, out, lanes=lanes, stream=stream)
            else:
                code = {"ticket_board": svdag.TABLE_LAYOUT_TICKET_BOARD, "atomic64": svdag.TABLE_LAYOUT_ATOMIC64,
                        "acceleration": svdag.TABLE_LAYOUT_ACCELERATION,
                        "individual_chaining": svdag.TABLE_LAYOUT_INDIVIDUAL_CHAINING}[layout]
                tbl = svdag.AltHashTable(dag, code, k, buckets, 2 * (n0 + n1))
                add = lambda kd, n, out: tbl.add(kd, n, out, lanes=lanes, stream=stream)
                find = lambda kd, n, out: tbl.find(kd, n, out, lanes=lanes, stream=stream)
            out0 = torch.empty(n0, dtype=torch.int32, device="cuda")
            out1 = torch.empty(n1, dtype=torch.int32, device="cuda")
            outs = torch.empty(ns, dtype=torch.int32, device="cuda")
            # untimed warm-up on a small table of the same layout and form: the first launch of a kernel
            # also loads it (lazy module loading)
            if layout == "compact":
                warm = dag.create_table(svdag.KIND_NODE, per_size // 64 + 1)
                warm.add(d_more, offs[n1], min(n1, 4096), k * min(n1, 4096), out1, lanes=lanes, stream=stream)
                warm.find(d_more, offs[n1], min(n1, 4096), k * min(n1, 4096), out1, lanes=lanes, stream=stream)
            else:
                warm = svdag.AltHashTable(dag, code, k, 64, 8192)
                warm.add(d_more, min(n1, 4096), out1, lanes=lanes, stream=stream)
                warm.find(d_more, min(n1, 4096), out1, lanes=lanes, stream=stream)
            stream.synchronize()
            warm.destroy()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(14)]
            torch.cuda.synchronize()
            found = {}
            with torch.cuda.stream(stream):
                ev[0].record(stream)
                add(d_init, n0, out0)
                ev[1].record(stream)
                for j, pct in enumerate(searches):
                    ev[2 + 2 * j].record(stream)
                    find(searches[pct][0], ns, outs)
                    ev[3 + 2 * j].record(stream)
                    found[pct] = (outs != -1).sum()
                ev[12].record(stream)
                add(d_more, n1, out1)
                ev[13].record(stream)
            stream.synchronize()
            if layout == "compact":
                dag.sync()
            else:
                tbl.sync(stream)
            r = {"layout": layout, "lanes": lanes, "bulk_add1_ms": ev[0].elapsed_time(ev[1]),
                 "bulk_add2_ms": ev[12].elapsed_time(ev[13])}
            for j, pct in enumerate(searches):
                r[f"search_hit{pct}_ms"] = ev[2 + 2 * j].elapsed_time(ev[3 + 2 * j])
                assert int(found[pct]) == searches[pct][1], (layout, lanes, pct, int(found[pct]))
            assert bool((out0 != -1).all()) and bool((out1 != -1).all()), (layout, lanes)
            r["bulk_add1_mitems_s"] = n0 / r["bulk_add1_ms"] / 1e3
            r["search_hit50_mitems_s"] = ns / r["search_hit50_ms"] / 1e3
            # algorithmic bytes, the same fixed formulas for every layout: add 4k + 32 + 4k + 4,
            # find 4k + 32 + 4k*hit + 4 per key of k words
            add_b = n0 * (8 * k + 36)
            r["bulk_add1_gbs"] = add_b / r["bulk_add1_ms"] / 1e6
            r["bulk_add1_frac"] = r["bulk_add1_gbs"] / peak
            for pct in searches:
                find_b = ns * (4 * k + 36) + searches[pct][1] * 4 * k
                r[f"search_hit{pct}_gbs"] = find_b / r[f"search_hit{pct}_ms"] / 1e6
            r["search_hit50_frac"] = r["search_hit50_gbs"] / peak
            st = tbl.stats(stream) if layout != "compact" else tbl.stats()
            r["items"], r["slab_bytes"] = int(st.items), int(st.bytes)
            results.append(r)
            tbl.destroy()
    dag.free()
    print(json.dumps({"mode": "hashmap", "item_words": k, "initial_items": n0, "insert_items": n1, "search_items": ns,
                      "buckets": buckets, "hbm_peak_gbs": peak, "peak": peak_kind, "results": results}))


def run_mode_c0(args):
    """Depth-10 terrain, then K sphere edits of the C0 stream each followed by a 256x256 frame."""
    import torch

    import svdag
    import svdag.workloads as w

    edits = w.c0_edits(max(args.warmup + args.steps, 64))
    dag = svdag.MyGPUHashDAG(w.C0_LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30, phase_kernels=args.phase_kernels,
                             persistent=args.persistent)
    dag.build_terrain(**w.C0_TERRAIN)
    params = svdag.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), C0_FRAME, C0_FRAME)
    hits = torch.empty(C0_FRAME * C0_FRAME * 68, dtype=torch.uint8, device="cuda")
    te, tt = [], []
    for i in range(args.warmup + args.steps):
        tool, mat, c, r = edits[i % len(edits)]
        e = w.make_edit(tool, mat, c, r)
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
    dag.sync()
    print(json.dumps({"edit_ms_p50": pct(te, 50), "edit_ms_p99": pct(te, 99), "trace_ms_p50": pct(tt, 50)}))


def run_mode_c2(args):
    """The at-scale sequence (carve, copy, noise paint) timed per edit with its phase timestamps."""
    import torch

    import svdag
    import svdag.workloads as w

    t0 = time.perf_counter()
    dag, terrain = make_scene(svdag, w, args.levels, phase_kernels=args.phase_kernels, pool_gb=args.pool_gb,
                              persistent=args.persistent)
    build_s = time.perf_counter() - t0
    out = []
    # capture every tool's graph before timing: a tiny edit of each kind far from the sequence, undone
    for e in w.c2_edits(args.levels, terrain):
        tiny = w.make_edit(e.tool, 0, (3.0, 3.0, 3.0), 1.0, src=(3.0, 3.0, 3.0), dst=(5.0, 3.0, 3.0))
        dag.edit(tiny)
        dag.undo()
    torch.cuda.synchronize()
    prof = profiled()
    prof.__enter__()
    for e in w.c2_edits(args.levels, terrain):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        dag.edit(e)
        b.record()
        torch.cuda.synchronize()
        st = dag.last_edit_stats()
        pt = [] if args.phase_kernels else dag.last_edit_phase_times()
        out.append({"tool": int(e.tool), "ms": a.elapsed_time(b), "status": int(st.status),
                    "edited_mvox": st.edited_voxels / 1e6, "svo_items": int(sum(st.svo_nodes)), "new_items": int(st.new_items),
                    "phase_us": [round(float(pt[i + 1] - pt[i]) / 1e3, 1) for i in range(len(pt) - 1)]})
    prof.__exit__()
    dag.free()
    print(json.dumps({"levels": args.levels, "build_s": build_s, "edits": out}))


def run_mode_trace(args):
    """1920x1080 primary-ray frames of the at-scale scene (at --levels), CUDA-event timed."""
    import torch

    import svdag
    import svdag.workloads as w

    dag, _ = make_scene(svdag, w, args.levels, pool_gb=args.pool_gb)
    cam = c2_camera(svdag, args.levels)
    tracer = svdag.DAGTracer(cam.width, cam.height)
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        tracer.resolve_paths(cam, dag, stream=stream.cuda_stream)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for a, b in ev:
        a.record(stream)
        tracer.resolve_paths(cam, dag, stream=stream.cuda_stream)
        b.record(stream)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    hits = tracer.hits_numpy()
    dag.free()
    print(json.dumps({"levels": args.levels, "frame_ms_p50": pct(ms, 50), "mrays_s": cam.width * cam.height / pct(ms, 50) / 1e3,
                      "hit_fraction": float((hits["material"] != 255).mean())}))


def c3_compare(svdag, w, torch, levels, edits):
    """The edits through the plain per-edit path and through one batch (the persistent kernel for small
    edits, subtree groups for runs of small edits in disjoint nodes), each on its own copy of the
    scene; the stored item sets must be equal."""
    res, items = {}, {}
    for name in ("plain", "batched"):
        dag, _ = make_scene(svdag, w, levels, persistent=name == "batched")
        stream = torch.cuda.Stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with profiled():
            a.record(stream)
            if name == "plain":
                for e in edits:
                    dag.edit(e, stream=stream.cuda_stream)
            else:
                dag.edit_batch(edits, stream=stream.cuda_stream)
            b.record(stream)
        torch.cuda.synchronize()
        dag.sync()
        res[name] = a.elapsed_time(b)
        items[name] = [dag.table(l).stats().items for l in range(levels - 1)]
        dag.free()
    return {"edits": len(edits), "plain_ms": res["plain"], "batched_ms": res["batched"],
            "items_equal": items["plain"] == items["batched"]}


def run_mode_c3(args):
    """256 edits of uneven footprint (radius log-uniform up to 4096 at depth 17), and 256 small edits
    of the same mix (radius 4..16) scattered over the surface: the batched form against the plain
    per-edit path."""
    import torch

    import svdag
    import svdag.workloads as w

    terrain = make_terrain(w, args.levels)
    out = {}
    if args.c3_set in ("both", "c3"):
        c3 = w.c3_edits(levels=args.levels, terrain=terrain, rmax=4096.0 * (1 << args.levels) / 131072)
        out = c3_compare(svdag, w, torch, args.levels, c3)
    if args.c3_set in ("both", "small"):
        small = w.c3_edits(levels=args.levels, terrain=terrain, rmax=16.0, seed=5)
        out["small_scattered"] = c3_compare(svdag, w, torch, args.levels, small)
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--mode", default="serve", choices=["serve", "c0", "c2", "c3", "hash", "hashmap", "trace"],
                    help="serve = the benchmark line; the others run one sub-workload (profiling)")
    ap.add_argument("--rate", type=float, default=1000.0, help="edit arrivals per second")
    ap.add_argument("--window", type=float, default=0.5, help="seconds of the stream per step")
    ap.add_argument("--sweep", default="50,200,500,2000", help="other offered loads (edits/s) served and plain")
    ap.add_argument("--levels", type=int, default=17)
    ap.add_argument("--phase-kernels", action="store_true", help="one launch per edit phase (profiling)")
    ap.add_argument("--persistent", action="store_true", help="small edits in the persistent cooperative kernel")
    ap.add_argument("--pool-gb", type=float, default=0.0, help="pool size of the c2 mode's scene (0 = by depth)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-hash", action="store_true")
    ap.add_argument("--no-batching", action="store_true", help="skip the batched-form comparison on small edits")
    ap.add_argument("--c3-set", default="both", choices=["both", "c3", "small"], help="--mode c3: which edit sets")
    ap.add_argument("--hash-keys", type=int, default=1 << 24)
    ap.add_argument("--hash-lanes", type=int, default=1)
    ap.add_argument("--hash-lf", type=int, default=16)
    ap.add_argument("--hash-reps", type=int, default=3)
    ap.add_argument("--hash-pool", type=int, default=6 << 30)
    ap.add_argument("--hashmap-initial", type=int, default=8 << 20)
    ap.add_argument("--hashmap-insert", type=int, default=1 << 20)
    ap.add_argument("--hashmap-search", type=int, default=1 << 20)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "hash":
        run_mode_hash(args)
    elif args.mode == "hashmap":
        run_mode_hashmap(args)
    elif args.mode == "c0":
        run_mode_c0(args)
    elif args.mode == "c2":
        run_mode_c2(args)
    elif args.mode == "c3":
        run_mode_c3(args)
    elif args.mode == "trace":
        run_mode_trace(args)
    else:
        run_serve(args)


if __name__ == "__main__":
    main()
