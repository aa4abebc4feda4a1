"""Octree dump/load (DumpSVOAsBinary / Constrcut(data)) and image files of
the tracers on the GPU.

The dump of a guided tracer's octree must be the reference's byte layout of
the state the tracer exports (restated independently in the oracle
package), must load back to the same bytes, and a tracer started from a
dump must render the next frame exactly as the tracer that wrote it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPTS = {"Samples": 1, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
        "DirectLightMIS": 0, "Seed": 3, "OctreeLevel": 6, "MinRayBinLevel": 3,
        "BinRayCount": 64}
HEADER = 48


def _wfpg(system, scene, opts=OPTS):
    from meturay_b200 import GPUScene, WFPGTracer
    g = GPUScene(system, scene)
    g.construct_accelerators()
    t = WFPGTracer(system, g)
    t.set_options(opts)
    return g, t


def _scene():
    from meturay_b200 import scenes
    return scenes.cornell(seed=2, width=40, height=32, mixed=True)


def _sections(ex):
    """Byte ranges of the node and leaf bin-info arrays in a dump."""
    N, U = ex["nodes_count"], ex["leaves"]
    nb = HEADER + 8 * N
    lb = nb + 2 * N + 4 * U
    return (nb, nb + 2 * N), (lb, lb + 2 * U)


def test_dump_layout_matches_the_restatement(system, oracle):
    g, t = _wfpg(system, _scene())
    for _ in range(3):
        t.render_frame()
    data = t.dump_svo()
    ex = t.export_svo()
    (a0, a1), (b0, b1) = _sections(ex)
    node_bins = np.frombuffer(data[a0:a1], np.uint16)
    leaf_bins = np.frombuffer(data[b0:b1], np.uint16)
    ref = oracle.svo_dump_bytes(ex, node_bins, leaf_bins)
    assert len(data) == len(ref) and data == ref
    # bin info: mark bit 15 and a count capped at 15 bits
    assert ((node_bins & 0x7FFF) <= 0x7FFF).all() and (leaf_bins >= 0).all()
    assert np.frombuffer(data[:24], np.float32).tolist() == [*ex["lo"], *ex["hi"]]


def test_load_round_trip_and_next_frame(system):
    scene = _scene()
    _, a = _wfpg(system, scene)
    for _ in range(3):
        a.render_frame()
    d3 = a.dump_svo()
    ex_a = a.export_svo()
    _, b = _wfpg(system, scene, dict(OPTS, OctreeLevel=4))  # the dump decides the octree
    b.load_svo(d3)
    assert b.dump_svo() == d3
    ex_b = b.export_svo()
    for k in ("nodes", "leaf_parents", "level_offsets", "leaf_normals", "node_normals",
              "leaf_cnt", "leaf_avg", "node_avg"):
        assert np.array_equal(ex_a[k], ex_b[k]), k
    assert ex_b["resolution"] == ex_a["resolution"] and not ex_b["leaf_codes"].any()
    # the dump carries N bytes of the node guiding factors; the shadow-ray
    # counters start again at zero
    N = ex_a["nodes_count"]
    assert ex_b["node_factor"].tobytes()[:N] == ex_a["node_factor"].tobytes()[:N]
    assert ex_a["leaf_shadow"].any() and not ex_b["leaf_shadow"].any()
    # the next frame reads only the averages, which load back exactly
    a.render_frame()
    b.set_options({"Frame": 3})
    b.render_frame()
    assert np.array_equal(a.sample_radiance(), b.sample_radiance())


def test_initial_svo_option_and_periodic_dumps(system, tmp_path):
    scene = _scene()
    name = str(tmp_path / "svo.bin")
    opts = dict(OPTS, PGDumpDataStruct=1, PGDataStructDumpIntervalExp=2,
                PGDataStructDumpName=name)
    _, a = _wfpg(system, scene, opts)
    dumps = {}
    for frame in range(1, 6):
        a.render_frame()
        dumps[frame] = a.dump_svo()
    files = sorted(p.name for p in tmp_path.iterdir())
    assert files == ["1_svo.bin", "2_svo.bin", "4_svo.bin"]
    for k in (1, 2, 4):
        assert (tmp_path / f"{k}_svo.bin").read_bytes() == dumps[k]
    _, c = _wfpg(system, scene, dict(OPTS, InitialSVO=str(tmp_path / "4_svo.bin")))
    c.generate_work()
    assert c.dump_svo() == dumps[4]


def test_bad_dumps_are_rejected(system):
    import meturay_b200 as m
    scene = _scene()
    _, a = _wfpg(system, scene)
    a.render_frame()
    good = a.dump_svo()
    ex = a.export_svo()
    N = ex["nodes_count"]
    _, b = _wfpg(system, scene)

    def patched(offset, fmt, value):
        d = bytearray(good)
        d[offset:offset + np.dtype(fmt).itemsize] = np.array([value], fmt).tobytes()
        return bytes(d)

    cases = [
        (good[:-1], "size mismatch"),
        (patched(24, "<u4", 48), "resolution"),                          # not a power of two
        (patched(HEADER + 8 * (N - 1), "<u8",
                 (int(ex["nodes"][N - 1]) & ~0x7FFFFFF) | 0x7FFFFFF), "children"),
        (patched(HEADER + 8 * N + 2 * N, "<u4", 0), "leaf parent"),      # leaf 0's parent = root
        (patched(44, "<u4", 3), "size mismatch"),                        # level offset count
    ]
    for data, needle in cases:
        with pytest.raises(m.MrbError, match=needle):
            b.load_svo(data)
    # the tracer is still usable afterwards
    b.load_svo(good)
    b.render_frame()


def test_tracer_image_files(system, tmp_path):
    import meturay_b200 as m
    from meturay_b200 import imageio
    _, t = _wfpg(system, _scene())
    t.attach_recon_filter(m.ReconFilter("Tent", 1.0))
    for _ in range(2):
        t.render_frame()
    img = t.image()
    est = np.where(img[..., 3:] != 0, img[..., :3] / np.where(img[..., 3:] != 0, img[..., 3:], 1),
                   0).astype(np.float32)
    for ext in ("exr", "pfm"):
        f = tmp_path / f"t.{ext}"
        t.write_image(f)
        assert np.array_equal(imageio.read_image(f), est)
    im = m.ImageMemory(16, 8, 4)
    f = m.ReconFilter("Box", 0.0)
    import torch
    v = torch.ones((4, 4), device="cuda") * 3
    c = torch.tensor([[0.5, 0.5], [0.5, 0.5], [3.5, 2.5], [15.5, 7.5]], device="cuda")
    f.filter_to_img(im, v, c, 4)
    im.write(tmp_path / "im.exr")
    r = imageio.read_image(tmp_path / "im.exr")
    assert r.shape == (8, 16, 4) and np.all(r[0, 0] == 3) and np.all(r[7, 15] == 3)
    assert np.all(r[1, 1] == 0)
