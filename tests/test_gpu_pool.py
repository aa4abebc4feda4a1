"""Wavefront pool (continuous batching of render jobs) on the GPU.

A job renders the same samples alone, in any mix of other jobs and as the
single PathTracer does (same scene, camera, options, seed and frames):
every random number is keyed by the job's own sample index, frame and seed.
Tolerance: relative mean error of the image below 1e-4 (the float atomic
accumulation of a sample's contributions may add in another order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4


def _rel(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))


def _scene(system, seed, tris=None, w=48, h=40, mixed=False):
    from meturay_b200 import GPUScene, scenes
    g = GPUScene(system, scenes.cornell(seed=seed, width=w, height=h, mixed=mixed,
                                        triangles=tris))
    g.construct_accelerators()
    return g


def _tracer_image(system, g, job):
    from meturay_b200 import PathTracer
    t = PathTracer(system, g)
    t.set_resolution(job.width, job.height)
    t.set_options({"Samples": job.samples, "MaxDepth": job.max_depth,
                   "NextEventEstimation": job.nee, "RussianRouletteStart": job.rr_start,
                   "DirectLightMIS": job.mis, "Seed": job.seed})
    for _ in range(job.frames):
        t.generate_work()
        while t.render():
            pass
        t.finalize()
    return t.image()


def _run(pool, jobs):
    return pool.run(jobs)


def test_job_alone_equals_the_path_tracer(system):
    from meturay_b200 import Job, WavefrontPool
    g = _scene(system, 3, mixed=True)
    job = Job(g, 48, 40, samples=2, frames=3, max_depth=5, seed=7, mis=1)
    pool = WavefrontPool(system, capacity=1 << 16, max_depth=6)
    img = _run(pool, [job])[0]
    ref = _tracer_image(system, g, job)
    assert img.shape == ref.shape and np.all(img[..., 3] == 3.0)
    assert _rel(img[..., :3], ref[..., :3]) < REL_TOL


def test_same_result_alone_and_in_the_mix(system):
    from meturay_b200 import Job, WavefrontPool
    g1 = _scene(system, 1)
    g2 = _scene(system, 2, tris=20000, mixed=True)
    g3 = _scene(system, 5, tris=3000)
    a = Job(g1, 40, 32, samples=1, frames=4, max_depth=5, seed=11)
    others = [Job(g2, 64, 48, samples=2, frames=2, max_depth=6, seed=3, mis=1),
              Job(g3, 24, 24, samples=1, frames=6, max_depth=3, seed=5, nee=0),
              Job(g1, 32, 32, samples=3, frames=1, max_depth=4, seed=9)]
    pool = WavefrontPool(system, capacity=1 << 16, max_depth=6)
    alone = _run(pool, [a])[0]
    mixed = _run(pool, others[:2] + [a] + others[2:])
    assert _rel(mixed[2][..., :3], alone[..., :3]) < REL_TOL
    assert np.array_equal(mixed[2][..., 3], alone[..., 3])
    # the others match their own lone renders too
    for j, img in zip(others[:2] + others[2:], mixed[:2] + mixed[3:]):
        assert _rel(img[..., :3], _run(pool, [j])[0][..., :3]) < REL_TOL
    st = pool.stats()
    assert st["hbm_used"] == 0 and st["rays"] > 0


def test_admission_by_hbm_budget_and_round_robin(system):
    from meturay_b200 import Job, WavefrontPool
    g = _scene(system, 4)
    img_bytes = 64 * 48 * 16
    # room for two images at a time; one iteration holds one 64x48x2^2 frame
    pool = WavefrontPool(system, capacity=64 * 48 * 4, max_depth=5, hbm_budget=2 * img_bytes)
    jobs = [Job(g, 64, 48, samples=2, frames=2, max_depth=5, seed=s) for s in range(5)]
    ids = [pool.submit(j) for j in jobs]
    seen_active, order = [], []
    while True:
        f, a, q = pool.step()
        st = pool.stats()
        assert st["hbm_used"] <= 2 * img_bytes
        seen_active.append(a)
        for jid in ids:
            if jid not in order and pool.status(jid)[0] == 2:
                order.append(jid)
                pool.image(jid)   # release: frees the budget for the queue
        if a == 0 and q == 0:
            break
    assert max(seen_active) <= 2 and sorted(order) == ids
    assert order[:2] == ids[:2]          # first come, first served
    # each job still renders what it renders alone
    alone = _run(WavefrontPool(system, capacity=1 << 16, max_depth=5), [jobs[4]])[0]
    pool2 = WavefrontPool(system, capacity=64 * 48 * 4, max_depth=5, hbm_budget=2 * img_bytes)
    imgs = _run(pool2, jobs)
    assert _rel(imgs[4][..., :3], alone[..., :3]) < REL_TOL


def test_launch_shapes_agree(system):
    from meturay_b200 import Job, WavefrontPool
    g = _scene(system, 6, tris=50000)
    job = Job(g, 40, 40, samples=2, frames=2, max_depth=5, seed=2)
    ref = None
    for block in (64, 128, 256):
        for stack in (64, 128, 0):  # 0: the octant child order
            pool = WavefrontPool(system, capacity=1 << 15, max_depth=5)
            pool.set_launch(block, stack)
            img = _run(pool, [job])[0]
            if ref is None:
                ref = img
            assert _rel(img[..., :3], ref[..., :3]) < REL_TOL


def test_pool_argument_errors(system):
    import meturay_b200 as m
    from meturay_b200 import Job, WavefrontPool
    g = _scene(system, 1)
    pool = WavefrontPool(system, capacity=1000, max_depth=4)
    with pytest.raises(m.MrbError, match="capacity"):
        pool.submit(Job(g, 64, 64, max_depth=4))         # one frame > capacity
    with pytest.raises(m.MrbError, match="max depth"):
        pool.submit(Job(g, 16, 16, max_depth=6))
    with pytest.raises(m.MrbError):
        pool.set_launch(96, 64)
    with pytest.raises(m.MrbError):
        WavefrontPool(system, capacity=0)
    small = WavefrontPool(system, capacity=1 << 12, max_depth=4, hbm_budget=1000)
    with pytest.raises(m.MrbError, match="budget"):
        small.submit(Job(g, 16, 16, max_depth=4))
    jid = pool.submit(Job(g, 8, 8, max_depth=4))
    with pytest.raises(m.MrbError, match="not done"):
        pool.image(jid)
    pool.drain()
    assert pool.image(jid).shape == (8, 8, 4)


def test_autotune_picks_a_measured_config(system):
    from meturay_b200 import Job
    from meturay_b200.pool import autotune
    gs = [_scene(system, s, tris=t) for s, t in ((1, 2000), (2, 30000))]
    jobs = [Job(g, 64, 64, samples=2, max_depth=4, seed=i) for i, g in enumerate(gs)]
    r = autotune(system, jobs, capacities=(1 << 14, 1 << 16), blocks=(64, 128), stacks=(64,),
                 max_depth=4, iterations=2)
    assert r["best"] in r["table"] and len(r["table"]) == 4
    assert all(row["mrays_s"] > 0 for row in r["table"])
