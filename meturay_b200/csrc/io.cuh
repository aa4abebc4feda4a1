// Files of the guided tracer and of images: the octree's binary dump
// (AnisoSVOctreeCPU::DumpSVOAsBinary / Constrcut(data), AnisoSVO.cu:1190-1413,
// 1555-1697) and headless image files (OpenEXR scanline, PFM) in place of
// the reference's FreeImage/OpenEXR image writer (ImageIO/ImageIO.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "svo.cuh"

namespace mrb {

// Bytes of the dump of an octree with these counts.
size_t svo_dump_size(uint32_t nodeCount, uint32_t leafCount, uint32_t levelOffsetCount);
// Serialise the octree and its radiance payload (synchronises the stream).
int svo_dump(const SvoResult& v, const SvoParams& P, std::vector<uint8_t>& out, cudaStream_t st);
// Rebuild an octree from a dump; out must be empty.  The dump carries no
// leaf Morton codes, run starts or light keys: those stay null.
int svo_load(const uint8_t* data, size_t size, SvoParams& P, SvoResult& out, cudaStream_t st);

// Images: rows bottom to top as the tracers produce them (row 0 = bottom).
// channels 1 (Y / grey), 3 (RGB) or 4 (RGBA).
int write_pfm(const std::string& path, const float* pixels, uint32_t w, uint32_t h,
              uint32_t channels);
int write_exr(const std::string& path, const float* pixels, uint32_t w, uint32_t h,
              uint32_t channels, bool half);
// Readers for the same files (EXR: uncompressed scanline files only).
// pixels receive w*h*channels floats, rows bottom to top.
int read_pfm(const std::string& path, std::vector<float>& pixels, uint32_t& w, uint32_t& h,
             uint32_t& channels);
int read_exr(const std::string& path, std::vector<float>& pixels, uint32_t& w, uint32_t& h,
             uint32_t& channels);
// Case-insensitive file-extension test.
bool ends_with(const std::string& s, const char* suffix);
// sums / counts per pixel (0 where a count is 0), first outChannels of
// channels, to .exr (FLOAT) or .pfm by the path's extension.
int write_averaged(const std::string& path, const float* sums, const float* counts,
                   uint32_t countStride, uint32_t width, uint32_t height, uint32_t channels,
                   uint32_t outChannels);

}  // namespace mrb
