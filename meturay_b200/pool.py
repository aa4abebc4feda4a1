"""Wavefront pool: continuous batching of render jobs (``mrb_pool_*``).

Jobs of different scenes, resolutions and sample counts share one
device-resident wavefront; the native pool admits them by free HBM, renders
one frame of every admitted job per iteration (one captured CUDA graph) and
finishes each after its frame count.  ``serve`` replays a stream of arrivals
against the pool's clock and reports per-job latency; ``autotune`` picks the
wavefront size and the traversal launch shape for a workload.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import MrbError, PoolJob, check, lib
from .tracer import GPUScene, TracerSystem, make_camera

__all__ = ["WavefrontPool", "Job", "serve", "autotune", "JOB_QUEUED", "JOB_ACTIVE", "JOB_DONE"]

JOB_QUEUED, JOB_ACTIVE, JOB_DONE = 0, 1, 2


@dataclass
class Job:
    """A render job: the scene's own camera unless one is given."""
    scene: GPUScene
    width: int
    height: int
    samples: int = 1          # s -> s*s per pixel per frame
    frames: int = 1           # spp = frames * s*s
    max_depth: int = 5
    rr_start: int = 3
    nee: int = 1
    mis: int = 0
    seed: int = 1
    camera: dict | None = None
    meta: dict = field(default_factory=dict)


class WavefrontPool:
    def __init__(self, system: TracerSystem, capacity: int = 1 << 20, max_depth: int = 8,
                 hbm_budget: int = 0):
        h = C.c_void_p()
        check(lib.mrb_pool_create(system._h, int(capacity), int(max_depth), int(hbm_budget),
                                  C.byref(h)))
        self._h = h
        self.system = system
        self.capacity = int(capacity)
        self.max_depth = int(max_depth)
        self._jobs: dict[int, Job] = {}

    def close(self):
        if getattr(self, "_h", None):
            lib.mrb_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_launch(self, block: int = 128, stack: int = 128):
        check(lib.mrb_pool_set_launch(self._h, int(block), int(stack)))

    def submit(self, job: Job) -> int:
        d = PoolJob()
        d.camera = make_camera(job.camera or job.scene.scene.camera)
        d.width, d.height, d.samples, d.frames = job.width, job.height, job.samples, job.frames
        d.max_depth, d.rr_start, d.nee, d.mis = job.max_depth, job.rr_start, job.nee, job.mis
        d.seed = job.seed
        jid = C.c_uint64()
        check(lib.mrb_pool_submit(self._h, job.scene._h, C.byref(d), C.byref(jid)))
        self._jobs[int(jid.value)] = job
        return int(jid.value)

    def step(self) -> tuple[int, int, int]:
        """One iteration: (finished, active, queued)."""
        f, a, q = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.mrb_pool_step(self._h, C.byref(f), C.byref(a), C.byref(q)))
        return int(f.value), int(a.value), int(q.value)

    def status(self, jid: int) -> tuple[int, int]:
        s, fr = C.c_uint32(), C.c_uint32()
        check(lib.mrb_pool_job_status(self._h, int(jid), C.byref(s), C.byref(fr)))
        return int(s.value), int(fr.value)

    def image(self, jid: int, release: bool = True) -> np.ndarray:
        job = self._jobs[jid]
        out = np.zeros((job.height, job.width, 4), np.float32)
        check(lib.mrb_pool_job_image(self._h, int(jid), out.ctypes.data, 1 if release else 0))
        if release:
            self._jobs.pop(jid, None)
        return out

    def stats(self) -> dict:
        rays, its = C.c_uint64(), C.c_uint64()
        used, budget = C.c_size_t(), C.c_size_t()
        check(lib.mrb_pool_stats(self._h, C.byref(rays), C.byref(its), C.byref(used),
                                 C.byref(budget)))
        return {"rays": int(rays.value), "iterations": int(its.value),
                "hbm_used": int(used.value), "hbm_budget": int(budget.value)}

    def drain(self, max_iterations: int = 1_000_000) -> list[int]:
        """Step until nothing is queued or active; the ids finished, in order."""
        done = []
        pending = set(self._jobs)
        for _ in range(max_iterations):
            f, a, q = self.step()
            if f:
                for jid in list(pending):
                    if self.status(jid)[0] == JOB_DONE:
                        done.append(jid)
                        pending.discard(jid)
            if a == 0 and q == 0:
                return done
            if a == 0 and q > 0:
                raise MrbError(-4, "pool: queued jobs wait for HBM that finished jobs still "
                                   "hold; fetch their images with release=True (or use run)")
        raise MrbError(-4, "pool: drain did not finish")

    def run(self, jobs: list[Job]) -> list[np.ndarray]:
        """Submit the jobs, step until all are done, fetching (and releasing)
        each image as its job finishes; the images in submission order."""
        ids = [self.submit(j) for j in jobs]
        images: dict[int, np.ndarray] = {}
        while len(images) < len(ids):
            f, a, q = self.step()
            if f:
                for jid in ids:
                    if jid not in images and self.status(jid)[0] == JOB_DONE:
                        images[jid] = self.image(jid, release=True)
            elif a == 0 and q == 0:
                raise MrbError(-4, "pool: jobs vanished before they finished")
        return [images[i] for i in ids]


def serve(pool: WavefrontPool, arrivals: list[tuple[float, Job]], keep_images: bool = False):
    """Replay (arrival time in seconds from now, job) pairs against the wall
    clock: each job is submitted once its time has come, the pool steps
    while there is work, and a job's latency runs from its arrival to the end
    of the iteration that finished it.  Returns per-job records."""
    order = sorted(range(len(arrivals)), key=lambda i: arrivals[i][0])
    t0 = time.perf_counter()
    nxt = 0
    live: dict[int, dict] = {}
    records = []
    while nxt < len(order) or live:
        now = time.perf_counter() - t0
        while nxt < len(order) and arrivals[order[nxt]][0] <= now:
            at, job = arrivals[order[nxt]]
            jid = pool.submit(job)
            live[jid] = {"index": order[nxt], "arrival": at, "job": job}
            nxt += 1
        if not live:
            time.sleep(max(0.0, min(arrivals[order[nxt]][0] - now, 0.01)))
            continue
        f, _, _ = pool.step()
        end = time.perf_counter() - t0
        if f:
            for jid in list(live):
                if pool.status(jid)[0] == JOB_DONE:
                    rec = live.pop(jid)
                    rec["finish"] = end
                    rec["latency"] = end - rec["arrival"]
                    img = pool.image(jid, release=True)
                    if keep_images:
                        rec["image"] = img
                    rec.pop("job")
                    records.append(rec)
    return sorted(records, key=lambda r: r["index"])


def _finish(pool: WavefrontPool, ids: list[int]):
    pool.drain()
    for jid in ids:
        if pool.status(jid)[0] == JOB_DONE:
            pool.image(jid, release=True)


def autotune(system: TracerSystem, jobs: list[Job], capacities=(1 << 16, 1 << 18, 1 << 20, 1 << 22),
             blocks=(64, 128, 256), stacks=(64, 128, 0), max_depth: int = 8,
             iterations: int = 3) -> dict:
    """Measure rays/s of `iterations` pool iterations over the given jobs for
    each wavefront size (camera samples per iteration; 2 rays each) and
    traversal launch shape (block size; stack of 64 or 128 entries for the
    sorted child order, 0 for the octant order), and return the fastest
    configuration with the table of all measured ones.  The jobs' frame
    counts are replaced so that every timed iteration has work."""
    from dataclasses import replace
    table = []
    best = None
    for cap in capacities:
        fits = [replace(j, frames=iterations + 1) for j in jobs
                if j.width * j.samples * j.height * j.samples <= cap]
        if not fits:
            continue
        try:
            pool = WavefrontPool(system, capacity=cap, max_depth=max_depth)
        except MrbError:
            continue
        for block in blocks:
            for stack in stacks:
                pool.set_launch(block, stack)
                ids = [pool.submit(j) for j in fits]
                pool.step()             # graph capture and the first frames
                r0 = pool.stats()["rays"]
                t = time.perf_counter()
                for _ in range(iterations):
                    pool.step()
                dt = time.perf_counter() - t
                r1 = pool.stats()["rays"]
                _finish(pool, ids)
                rate = (r1 - r0) / dt / 1e6
                row = {"capacity": cap, "block": block, "stack": stack, "mrays_s": rate}
                table.append(row)
                if best is None or rate > best["mrays_s"]:
                    best = row
        pool.close()
    return {"best": best, "table": table}
