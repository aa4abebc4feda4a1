"""Golden vectors of the reference's ProductSampler (TracerCUDA/
ProductSampler.cuh), for tests/test_oracle_golden.py.

The sampler is device code that takes its BxDF through the reference's
material system and its random numbers through a curand generator.  The
harness `oracle/_ref/libpsamp.so` (built by `make -C oracle psamp`
REF_ROOT=<MRay tree> from oracle/psamp/) runs the reference's own sampler
on a B200 with table stand-ins for both.  This script feeds it seeded
inputs and stores inputs and outputs:

    python tests/golden/make_golden_product.py [out.npz]

It needs a GPU and the prebuilt harness, not the MRay tree.  The file holds
the outputs and a digest of the inputs, which `inputs()` regenerates from
its seed.  Inputs:
- 12 radiance fields of 64x64 (the sampler's X = Y = 64, 8x8 product map):
  smooth lognormal fields, fields with a few bright blobs, and fields with
  single spikes (so that rejection sampling sometimes fails its 24 rounds);
- 48 rays per field, each with a table surface (RGB per product cell, a
  BxDF sample's uv and pdf, and a linear Pdf) and 96 uniforms per lane in
  [0, 0.999) (the sampler's CDF searches then never run past the last cell).
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent.parent
BINS, RAYS_PER_BIN, STREAM = 12, 48, 96
SURFACE_FLOATS = 198
MIS_RATIO = 0.5


def inputs(seed: int = 20251203):
    rng = np.random.default_rng(seed)
    fields = np.empty((BINS, 64, 64), np.float32)
    yy, xx = np.mgrid[0:64, 0:64].astype(np.float64)
    for b in range(BINS):
        f = rng.lognormal(-1.0, 0.6, (64, 64))
        if b % 3 == 1:     # bright blobs
            for _ in range(3):
                cx, cy, r = rng.uniform(0, 64), rng.uniform(0, 64), rng.uniform(2, 8)
                f += 40.0 * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * r * r))
        elif b % 3 == 2:   # spikes: one texel per product cell far above the rest
            f *= 1e-3
            for cy in range(8):
                for cx in range(8):
                    f[cy * 8 + rng.integers(8), cx * 8 + rng.integers(8)] += rng.uniform(50, 500)
        fields[b] = f.astype(np.float32)
    rays = BINS * RAYS_PER_BIN
    surf = np.empty((rays, SURFACE_FLOATS), np.float32)
    surf[:, :192] = rng.uniform(0.02, 1.0, (rays, 192))
    surf[:, 192:194] = rng.uniform(0.0, 0.999, (rays, 2))
    surf[:, 194] = rng.uniform(0.05, 3.0, rays)
    surf[:, 195] = rng.uniform(0.05, 0.5, rays)
    surf[:, 196:198] = rng.uniform(0.0, 0.5, (rays, 2))
    streams = rng.uniform(0.0, 0.999, (rays, 32, STREAM)).astype(np.float32)
    return fields, surf, streams


def digest(*arrays) -> bytes:
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


def run(fields, surf, streams, mult):
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libpsamp.so"))
    vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    lib.psamp_run.argtypes = [vp, u32, u32, vp, vp, u32, f32, f32, vp, vp, vp, vp, vp, vp]
    rays = BINS * RAYS_PER_BIN
    uv = np.zeros((rays, 2), np.float32)
    pdf = np.zeros(rays, np.float32)
    sel = np.zeros(rays, np.uint32)
    small = np.zeros((BINS, 64), np.float32)
    norm = np.zeros((BINS, 64), np.float32)
    draws = np.zeros((rays, 32), np.uint32)
    p = lambda a: a.ctypes.data_as(vp)
    rc = lib.psamp_run(p(fields), BINS, RAYS_PER_BIN, p(surf), p(streams), STREAM, MIS_RATIO, mult,
                       p(uv), p(pdf), p(sel), p(small), p(norm), p(draws))
    if rc:
        raise RuntimeError("psamp_run failed")
    if draws.max() > STREAM:
        raise RuntimeError(f"a lane drew {draws.max()} uniforms, more than the table's {STREAM}")
    return uv, pdf, sel, small, norm, draws


def main():
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else ROOT / "tests" / "golden" / "product_sampler_vectors.npz"
    fields, surf, streams = inputs()
    mult = np.float32(0.25) * np.float32(1.0 / np.pi)  # the octahedral map's 1/(4 pi)
    uv, pdf, sel, small, norm, draws = run(fields, surf, streams, float(mult))
    # the inputs are regenerated from the seed by the test; their digest
    # guards against a change of the generator
    np.savez_compressed(out, input_digest=np.frombuffer(digest(fields, surf, streams), np.uint8),
                        mis_ratio=np.float32(MIS_RATIO), mult=np.float32(mult),
                        rays_per_bin=np.uint32(RAYS_PER_BIN), uv=uv, pdf=pdf, sel=sel,
                        small=small, norm=norm, draws=draws)
    print(f"{out}: {len(pdf)} rays, {int(sel.sum())} BxDF-selected, draws max {int(draws.max())}")


if __name__ == "__main__":
    main()
