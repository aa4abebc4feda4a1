"""Host-side checks that need no GPU: the C-ABI library loads and exports
every entry point include/mrb200.h declares, host-only entry points behave,
errors come back as status codes, and the scene generators are deterministic."""
import ctypes as C

import numpy as np
import pytest


def test_library_exports_every_declared_symbol():
    from meturay_b200 import _lib
    names = _lib.exported_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(_lib.lib, n)]
    assert not missing, missing


def test_oracle_library_exports():
    from oracle import oracle as o
    for n in ("oracle_render", "oracle_trace", "oracle_lbvh_build", "oracle_partition",
              "oracle_build_tbn", "oracle_probe", "oracle_philox4x32"):
        assert hasattr(o.lib, n)


def test_camera_frame_matches_pinhole_construction():
    import meturay_b200 as m
    cam = m.scenes.cornell(1).camera
    f = m.camera_frame(cam).astype(np.float64)
    pos, bl, right, up, size = f[0:3], f[3:6], f[6:9], f[9:12], f[12:14]
    assert np.allclose(pos, cam["position"])
    assert abs(np.linalg.norm(right) - 1) < 1e-6 and abs(np.linalg.norm(up) - 1) < 1e-6
    near = cam["near_far"][0]
    assert np.allclose(size, 2 * np.tan(np.array(cam["fov"]) / 2) * near, rtol=1e-5)
    # centre of the image plane lies on the gaze line at distance near
    centre = bl + right * size[0] / 2 + up * size[1] / 2
    g = np.array(cam["gaze"]) - np.array(cam["position"])
    g /= np.linalg.norm(g)
    assert np.allclose(centre, np.array(cam["position"]) + g * near, atol=1e-5)


def test_errors_are_status_codes():
    from meturay_b200._lib import MrbError, check, lib
    rc = lib.mrb_camera_frame(None, None)
    assert rc == -1
    with pytest.raises(MrbError):
        check(lib.mrb_radix_sort_pairs_u64(None, None, 10, 0, 70, 0, None, 0, None))
    assert "invalid" in lib.mrb_last_error().decode()


def test_system_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import meturay_b200 as m
    with pytest.raises(m.MrbError) as e:
        m.TracerSystem(0)
    assert e.value.code == -2


def test_sort_scratch_size_grows_with_count():
    from meturay_b200._lib import lib
    a = lib.mrb_radix_sort_temp_bytes(1000, 8, 0, 63)
    b = lib.mrb_radix_sort_temp_bytes(1 << 20, 8, 0, 63)
    assert 0 < a < b
    assert b >= (1 << 20) * 12


def test_scene_generators_deterministic():
    from meturay_b200 import scenes
    a, b = scenes.cornell(seed=4), scenes.cornell(seed=4)
    assert np.array_equal(a.positions, b.positions) and a.triangle_count == b.triangle_count
    assert 7000 < a.triangle_count < 8500
    c = scenes.cornell(seed=5)
    assert not np.array_equal(a.positions, c.positions)
    k = scenes.clusters(seed=1, n_clusters=20, tris_per_cluster=50)
    assert k.triangle_count == 20 * 50 + 8
    kinds = {m["type"] for m in k.materials}
    assert kinds == {1, 2, 3, 4}
    assert (k.positions.min(0) > -20).all() and (k.positions.max(0) < 120).all()


def test_mray_binding_compiles_against_the_reference_headers(tmp_path):
    """include/mray/GPUAccLBVHGroup.cuh implements MRay's GPUAcceleratorGroupI
    and GPUBaseAcceleratorI over the C ABI.  Compiled here with nvcc against
    the MRay sources the checker was built from (oracle/_ref/ref_root.txt,
    written by `make -C oracle ref`), with the flags MRay's TracerCUDA
    sources build with; both classes are instantiated so that every virtual
    member is compiled.  Compile only: nothing is linked into the library."""
    import subprocess
    from pathlib import Path
    root_file = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "ref_root.txt"
    if not root_file.exists():
        pytest.skip("the MRay sources are not present (checker built without them)")
    ref = Path(root_file.read_text().strip())
    if not (ref / "Source" / "TracerCUDA" / "GPUAcceleratorI.h").exists():
        pytest.skip("the MRay sources are not present here")
    inc = Path(__file__).resolve().parent.parent / "include"
    tu = tmp_path / "binding.cu"
    tu.write_text('#include "mray/GPUAccLBVHGroup.cuh"\n'
                  "GPUAcceleratorGroupI* make_group(const GPUPrimitiveGroupI& p) {\n"
                  "    return new mrb_mray::GPUAccLBVHGroup(p);\n}\n"
                  "GPUBaseAcceleratorI* make_base() { return new mrb_mray::GPUBaseAccLBVH(); }\n")
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-DMETU_CUDA", "-DFMT_HEADER_ONLY",
           "--expt-relaxed-constexpr", "--extended-lambda", "-rdc=true",
           "-gencode", "arch=compute_100a,code=sm_100a", "-I", str(ref / "Source"),
           "-I", str(ref / "Lib" / "Include"), "-I", str(inc), "-c", str(tu),
           "-o", str(tmp_path / "binding.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert (tmp_path / "binding.o").stat().st_size > 0
