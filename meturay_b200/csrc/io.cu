// Octree dump/load and image files (host code).
//
// Octree dump (DumpSVOAsBinary, AnisoSVO.cu:1555-1697; read back by
// Constrcut(data), AnisoSVO.cu:1190-1413), little endian, packed:
//   header   AABB (min xyz, max xyz: 6 f32), voxel resolution u32, leaf depth
//            u32, node count u32, leaf count u32, leaf voxel size f32, level
//            offset count u32                                       (48 B)
//   tree     nodes u64[N], node bin info u16[N], leaf parents u32[U],
//            leaf bin info u16[U], level node offsets u32[L]
//   payload  node average radiance f32x2[N], node normal+specular u32[N],
//            node guiding factor u8[N], leaf radiance sums f32x2[U], leaf
//            sample counts u32x2[U], leaf average radiance f32x2[U], leaf
//            normal+specular u32[U], leaf guiding factor u8[U]
// This core keeps bin words as 32-bit (mark bit 31, 31-bit count), leaf sums
// in 2^-24 fixed point and averages as half pairs; the dump converts each to
// the reference's field (16-bit bin info with mark bit 15 and a 15-bit
// count, FP32 sums, FP32 averages) and the load converts back.  The node
// guiding factor field holds N bytes of the binary16 node factors as they
// lie in memory (the first N / 2 factors: the reference copies N bytes of
// its half array); the leaf factor field stays 0 (the reference writes
// nothing there).  The load puts the N bytes back at the start of the half
// array, marks the rest NaN (no data) and starts the shadow-ray counters at
// zero; the next NormalizeAndFilterRadiance recomputes every factor.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/mrb200.h"
#include "io.cuh"
#include "svo_dev.cuh"

namespace mrb {

namespace {

constexpr size_t kSvoHeaderBytes = 48;

template <class T>
void put(std::vector<uint8_t>& out, size_t& off, const T* src, size_t count) {
    std::memcpy(out.data() + off, src, count * sizeof(T));
    off += count * sizeof(T);
}
template <class T>
void get(const uint8_t* data, size_t& off, T* dst, size_t count) {
    std::memcpy(dst, data + off, count * sizeof(T));
    off += count * sizeof(T);
}

int d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (!bytes) return 0;
    MRB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    return 0;
}
int h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (!bytes) return 0;
    MRB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return 0;
}

uint16_t bin_to_u16(uint32_t w) {
    const uint32_t count = w & 0x7FFFFFFFu;
    return static_cast<uint16_t>(((w & 0x80000000u) ? 0x8000u : 0u) |
                                 (count < 0x7FFFu ? count : 0x7FFFu));
}
uint32_t bin_from_u16(uint16_t b) {
    return ((b & 0x8000u) ? 0x80000000u : 0u) | (b & 0x7FFFu);
}

// 2^-24 fixed point <-> FP32: one rounding each way.  A float that came from
// a fixed-point sum is a multiple of 2^-24, so load(dump(x)) reproduces it.
float fixed_to_float(unsigned long long v) { return static_cast<float>(v) * 0x1p-24f; }
unsigned long long float_to_fixed(float f) {
    if (!(f > 0.0f)) return 0ull;  // negative, zero and NaN sums
    const double s = static_cast<double>(f) * 16777216.0;
    if (s >= 18446744073709551615.0) return ~0ull;
    return static_cast<unsigned long long>(std::nearbyint(s));
}

}  // namespace

size_t svo_dump_size(uint32_t N, uint32_t U, uint32_t L) {
    return kSvoHeaderBytes + size_t(N) * (8 + 2) + size_t(U) * (4 + 2) + size_t(L) * 4 +
           size_t(N) * (8 + 4 + 1) + size_t(U) * (8 + 8 + 8 + 4 + 1);
}

int svo_dump(const SvoResult& v, const SvoParams& P, std::vector<uint8_t>& out, cudaStream_t st) {
    const size_t N = v.nodeCount, U = v.leafCount, L = v.levelOffsets.size();
    out.assign(svo_dump_size(v.nodeCount, v.leafCount, static_cast<uint32_t>(L)), 0);
    std::vector<uint64_t> nodes(N);
    std::vector<uint32_t> nodeBin(N), nodeAvg(N), nodeNs(N), leafParents(U), leafBin(U),
        leafCnt(2 * U), leafAvg(U), leafNs(U);
    std::vector<unsigned long long> leafIrr(2 * U);
    std::vector<uint16_t> nodeFactor(N);
    if (d2h(nodes.data(), v.nodes, N * 8, st) || d2h(nodeBin.data(), v.nodeBin, N * 4, st) ||
        d2h(nodeAvg.data(), v.nodeAvg, N * 4, st) || d2h(nodeNs.data(), v.nodeNormSpec, N * 4, st) ||
        d2h(leafParents.data(), v.leafParents, U * 4, st) ||
        d2h(leafBin.data(), v.leafBin, U * 4, st) || d2h(leafCnt.data(), v.leafCnt, U * 8, st) ||
        d2h(leafAvg.data(), v.leafAvg, U * 4, st) ||
        d2h(leafNs.data(), v.leafNormSpec, U * 4, st) ||
        d2h(leafIrr.data(), v.leafIrr, U * 16, st) ||
        d2h(nodeFactor.data(), v.nodeFactor, N * 2, st))
        return MRB_E_CUDA;
    MRB_CUDA(cudaStreamSynchronize(st));
    size_t off = 0;
    put(out, off, P.lo, 3);
    put(out, off, P.hi, 3);
    const uint32_t head[4] = {P.res, P.depth, v.nodeCount, v.leafCount};
    put(out, off, head, 4);
    put(out, off, &P.leafVoxelSize, 1);
    const uint32_t levels = static_cast<uint32_t>(L);
    put(out, off, &levels, 1);
    put(out, off, nodes.data(), N);
    std::vector<uint16_t> b16(N > U ? N : U);
    for (size_t i = 0; i < N; i++) b16[i] = bin_to_u16(nodeBin[i]);
    put(out, off, b16.data(), N);
    put(out, off, leafParents.data(), U);
    for (size_t i = 0; i < U; i++) b16[i] = bin_to_u16(leafBin[i]);
    put(out, off, b16.data(), U);
    put(out, off, v.levelOffsets.data(), L);
    std::vector<float> f2(2 * (N > U ? N : U));
    for (size_t i = 0; i < N; i++) {
        f2[2 * i] = h2f(static_cast<uint16_t>(nodeAvg[i] & 0xFFFFu));
        f2[2 * i + 1] = h2f(static_cast<uint16_t>(nodeAvg[i] >> 16));
    }
    put(out, off, f2.data(), 2 * N);
    put(out, off, nodeNs.data(), N);
    std::memcpy(out.data() + off, nodeFactor.data(), N);  // N bytes of the half array
    off += N;
    for (size_t i = 0; i < 2 * U; i++) f2[i] = fixed_to_float(leafIrr[i]);
    put(out, off, f2.data(), 2 * U);
    put(out, off, leafCnt.data(), 2 * U);
    for (size_t i = 0; i < U; i++) {
        f2[2 * i] = h2f(static_cast<uint16_t>(leafAvg[i] & 0xFFFFu));
        f2[2 * i + 1] = h2f(static_cast<uint16_t>(leafAvg[i] >> 16));
    }
    put(out, off, f2.data(), 2 * U);
    put(out, off, leafNs.data(), U);
    off += U;  // leaf guiding factors: 0
    return off == out.size() ? 0 : MRB_E_STATE;
}

namespace {

int load_error(const char* what) {
    set_error("SVO load: %s", what);
    return MRB_E_ARG;
}

// The device code follows child, parent and level indices without bounds
// checks, so a dump is accepted only when every index lands in range.
int check_tree(const SvoParams& P, uint32_t N, uint32_t U, const std::vector<uint32_t>& lo,
               const std::vector<uint64_t>& nodes, const std::vector<uint32_t>& leafParents) {
    const uint32_t D = P.depth;
    if (lo.size() != D + 2u) return load_error("level offset count is not leaf depth + 2");
    if (lo[0] != 0 || lo[1] != 1) return load_error("level 0 must hold exactly the root");
    for (uint32_t l = 0; l + 1 < lo.size(); l++)
        if (lo[l + 1] < lo[l]) return load_error("level offsets decrease");
    if (lo[D] != N || uint64_t(lo[D + 1]) != uint64_t(N) + U)
        return load_error("level offsets disagree with the node and leaf counts");
    for (uint32_t l = 0; l < D; l++) {
        for (uint32_t i = lo[l]; i < lo[l + 1]; i++) {
            const uint64_t n = nodes[i];
            const uint32_t child = uint32_t(n & 0x7FFFFFFull);
            const uint32_t parent = uint32_t((n >> 27) & 0xFFFFFFFull);
            const uint32_t mask = uint32_t((n >> 55) & 0xFFull);
            const bool leafKids = (n >> 63) != 0;
            if (leafKids != (l + 1 == D)) return load_error("node child-type bit at the wrong level");
            if (l == 0 ? parent != kSvoInvalidParent : (parent < lo[l - 1] || parent >= lo[l]))
                return load_error("node parent outside the level above");
            const uint32_t kids = static_cast<uint32_t>(__builtin_popcount(mask));
            const uint64_t b = leafKids ? 0u : lo[l + 1], e = leafKids ? U : lo[l + 2];
            if (kids && (child < b || uint64_t(child) + kids > e))
                return load_error("node children outside the level below");
        }
    }
    for (uint32_t j = 0; j < U; j++)
        if (leafParents[j] < lo[D - 1] || leafParents[j] >= lo[D])
            return load_error("leaf parent outside the last node level");
    return 0;
}

}  // namespace

int svo_load(const uint8_t* data, size_t size, SvoParams& P, SvoResult& out, cudaStream_t st) {
    if (!data || size < kSvoHeaderBytes) return load_error("shorter than its header");
    size_t off = 0;
    SvoParams Q{};
    get(data, off, Q.lo, 3);
    get(data, off, Q.hi, 3);
    uint32_t head[4];
    get(data, off, head, 4);
    get(data, off, &Q.leafVoxelSize, 1);
    uint32_t L = 0;
    get(data, off, &L, 1);
    Q.res = head[0];
    Q.depth = head[1];
    const uint32_t N = head[2], U = head[3];
    if (Q.res < 2 || Q.res > 1024 || Q.depth < 1 || Q.depth > 10 || (1u << Q.depth) != Q.res)
        return load_error("voxel resolution is not 2^depth with depth in [1, 10]");
    for (int c = 0; c < 3; c++)
        if (!std::isfinite(Q.lo[c]) || !std::isfinite(Q.hi[c]) || !(Q.hi[c] > Q.lo[c]))
            return load_error("bounding box is empty or not finite");
    if (!std::isfinite(Q.leafVoxelSize) || !(Q.leafVoxelSize > 0.0f))
        return load_error("leaf voxel size is not positive");
    if (N == 0 || U == 0 || N >= (1u << 27) || U >= (1u << 27))
        return load_error("node or leaf count out of range");
    if (L > 64 || svo_dump_size(N, U, L) != size) {
        set_error("SVO load: Read SVO size mismatch (%zu bytes, the header implies %zu)", size,
                  svo_dump_size(N, U, L > 64 ? 0 : L));
        return MRB_E_ARG;
    }
    std::vector<uint64_t> nodes(N);
    std::vector<uint16_t> nodeBin16(N), leafBin16(U);
    std::vector<uint32_t> leafParents(U), levelOffsets(L), nodeNs(N), leafCnt(2 * size_t(U)),
        leafNs(U), nodeAvg(N), leafAvg(U), nodeBin(N), leafBin(U);
    std::vector<float> f2(2 * size_t(N > U ? N : U));
    std::vector<unsigned long long> leafIrr(2 * size_t(U));
    get(data, off, nodes.data(), N);
    get(data, off, nodeBin16.data(), N);
    get(data, off, leafParents.data(), U);
    get(data, off, leafBin16.data(), U);
    get(data, off, levelOffsets.data(), L);
    int r = check_tree(Q, N, U, levelOffsets, nodes, leafParents);
    if (r) return r;
    get(data, off, f2.data(), 2 * size_t(N));
    for (uint32_t i = 0; i < N; i++)
        nodeAvg[i] = uint32_t(f2h(f2[2 * i])) | (uint32_t(f2h(f2[2 * i + 1])) << 16);
    get(data, off, nodeNs.data(), N);
    std::vector<uint16_t> nodeFactor(N, kFactorNone);
    std::memcpy(nodeFactor.data(), data + off, N);
    off += N;
    get(data, off, f2.data(), 2 * size_t(U));
    for (size_t i = 0; i < 2 * size_t(U); i++) leafIrr[i] = float_to_fixed(f2[i]);
    get(data, off, leafCnt.data(), 2 * size_t(U));
    get(data, off, f2.data(), 2 * size_t(U));
    for (uint32_t i = 0; i < U; i++)
        leafAvg[i] = uint32_t(f2h(f2[2 * i])) | (uint32_t(f2h(f2[2 * i + 1])) << 16);
    get(data, off, leafNs.data(), U);
    off += U;  // leaf guiding factors
    for (uint32_t i = 0; i < N; i++) nodeBin[i] = bin_from_u16(nodeBin16[i]);
    for (uint32_t i = 0; i < U; i++) leafBin[i] = bin_from_u16(leafBin16[i]);

    SvoResult v{};
    v.leafCount = U;
    v.nodeCount = N;
    v.voxelCount = U;
    v.levelOffsets = levelOffsets;
    auto alloc = [&](void** p, size_t bytes) -> int {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            set_error("SVO load: cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
            return MRB_E_OOM;
        }
        return 0;
    };
    if ((r = alloc(reinterpret_cast<void**>(&v.nodes), size_t(N) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafParents), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafNormSpec), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.nodeNormSpec), size_t(N) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafIrr), size_t(U) * 16)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafCnt), size_t(U) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafAvg), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.nodeAvg), size_t(N) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafShadow), size_t(U) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&v.nodeFactor), size_t(N) * 2)) ||
        (r = alloc(reinterpret_cast<void**>(&v.leafBin), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.nodeBin), size_t(N) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&v.dLevelOffsets), size_t(L) * 4))) {
        svo_free(v);
        return r;
    }
    if (h2d(v.nodes, nodes.data(), size_t(N) * 8, st) ||
        h2d(v.leafParents, leafParents.data(), size_t(U) * 4, st) ||
        h2d(v.leafNormSpec, leafNs.data(), size_t(U) * 4, st) ||
        h2d(v.nodeNormSpec, nodeNs.data(), size_t(N) * 4, st) ||
        h2d(v.leafIrr, leafIrr.data(), size_t(U) * 16, st) ||
        h2d(v.leafCnt, leafCnt.data(), size_t(U) * 8, st) ||
        h2d(v.leafAvg, leafAvg.data(), size_t(U) * 4, st) ||
        h2d(v.nodeAvg, nodeAvg.data(), size_t(N) * 4, st) ||
        h2d(v.leafBin, leafBin.data(), size_t(U) * 4, st) ||
        h2d(v.nodeBin, nodeBin.data(), size_t(N) * 4, st) ||
        h2d(v.nodeFactor, nodeFactor.data(), size_t(N) * 2, st) ||
        cudaMemsetAsync(v.leafShadow, 0, size_t(U) * 8, st) != cudaSuccess ||
        h2d(v.dLevelOffsets, levelOffsets.data(), size_t(L) * 4, st)) {
        svo_free(v);
        return MRB_E_CUDA;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        set_error("SVO load: upload failed");
        svo_free(v);
        return MRB_E_CUDA;
    }
    out = v;
    P = Q;
    return 0;
}

// ---------------------------------------------------------------------------
// Images
// ---------------------------------------------------------------------------
namespace {

struct File {
    FILE* f = nullptr;
    explicit File(const std::string& path, const char* mode) { f = std::fopen(path.c_str(), mode); }
    ~File() {
        if (f) std::fclose(f);
    }
};

int io_error(const std::string& path, const char* what) {
    set_error("%s: %s", path.c_str(), what);
    return MRB_E_ARG;
}

bool read_all(const std::string& path, std::vector<uint8_t>& bytes) {
    File in(path, "rb");
    if (!in.f) return false;
    std::fseek(in.f, 0, SEEK_END);
    const long n = std::ftell(in.f);
    if (n < 0) return false;
    std::fseek(in.f, 0, SEEK_SET);
    bytes.resize(static_cast<size_t>(n));
    return n == 0 || std::fread(bytes.data(), 1, bytes.size(), in.f) == bytes.size();
}

int check_image_args(const std::string& path, const float* pixels, uint32_t w, uint32_t h,
                     uint32_t channels) {
    if (!pixels || w == 0 || h == 0 || (channels != 1 && channels != 3 && channels != 4))
        return io_error(path, "need pixels, a non-empty size and 1, 3 or 4 channels");
    if (uint64_t(w) * h > (uint64_t(1) << 30)) return io_error(path, "image too large");
    return 0;
}

template <class T>
void append(std::vector<uint8_t>& b, const T& v) {
    const size_t o = b.size();
    b.resize(o + sizeof(T));
    std::memcpy(b.data() + o, &v, sizeof(T));
}
void append_str(std::vector<uint8_t>& b, const char* s) {
    const size_t n = std::strlen(s) + 1;
    b.insert(b.end(), s, s + n);
}
void attr_head(std::vector<uint8_t>& b, const char* name, const char* type, int32_t size) {
    append_str(b, name);
    append_str(b, type);
    append(b, size);
}

}  // namespace

// Portable FloatMap: "PF" (RGB) or "Pf" (grey), little-endian scale -1,
// rows bottom to top -- the tracers' own row order.
int write_pfm(const std::string& path, const float* pixels, uint32_t w, uint32_t h,
              uint32_t channels) {
    int r = check_image_args(path, pixels, w, h, channels);
    if (r) return r;
    File out(path, "wb");
    if (!out.f) return io_error(path, "cannot open for writing");
    const uint32_t oc = channels == 1 ? 1 : 3;
    std::fprintf(out.f, "%s\n%u %u\n-1.0\n", oc == 1 ? "Pf" : "PF", w, h);
    std::vector<float> row(size_t(w) * oc);
    for (uint32_t y = 0; y < h; y++) {
        for (uint32_t x = 0; x < w; x++)
            for (uint32_t c = 0; c < oc; c++)
                row[size_t(x) * oc + c] = pixels[(size_t(y) * w + x) * channels + c];
        if (std::fwrite(row.data(), sizeof(float), row.size(), out.f) != row.size())
            return io_error(path, "short write");
    }
    return 0;
}

int read_pfm(const std::string& path, std::vector<float>& pixels, uint32_t& w, uint32_t& h,
             uint32_t& channels) {
    std::vector<uint8_t> b;
    if (!read_all(path, b)) return io_error(path, "cannot read");
    size_t p = 0;
    auto token = [&](std::string& t) {
        while (p < b.size() && std::isspace(b[p])) p++;
        t.clear();
        while (p < b.size() && !std::isspace(b[p])) t.push_back(static_cast<char>(b[p++]));
        return !t.empty();
    };
    std::string magic, sw, sh, ss;
    if (!token(magic) || !token(sw) || !token(sh) || !token(ss) || p >= b.size())
        return io_error(path, "truncated PFM header");
    p++;  // the single whitespace after the scale
    if (magic != "PF" && magic != "Pf") return io_error(path, "not a PFM file");
    channels = magic == "PF" ? 3 : 1;
    char* end = nullptr;
    const unsigned long lw = std::strtoul(sw.c_str(), &end, 10);
    const unsigned long lh = std::strtoul(sh.c_str(), &end, 10);
    const double scale = std::strtod(ss.c_str(), &end);
    if (lw == 0 || lh == 0 || lw * lh > (1ul << 30) || scale == 0.0)
        return io_error(path, "bad PFM size or scale");
    w = static_cast<uint32_t>(lw);
    h = static_cast<uint32_t>(lh);
    const size_t n = size_t(w) * h * channels;
    if (b.size() - p < n * 4) return io_error(path, "truncated PFM data");
    pixels.resize(n);
    std::memcpy(pixels.data(), b.data() + p, n * 4);
    if (scale > 0.0)  // big endian
        for (float& v : pixels) {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            u = __builtin_bswap32(u);
            std::memcpy(&v, &u, 4);
        }
    return 0;
}

// OpenEXR, single-part scanline, NO_COMPRESSION, one line per block, as
// described by the OpenEXR file-layout document: magic 20000630, version
// 2, the required header attributes, a 64-bit offset per line and the lines
// (y, byte count, then each channel's samples in the channel list's
// alphabetical order).  Channels are R, G, B (, A) or Y for one channel, in
// FLOAT or HALF with pLinear set, as ImageIO::WriteAsEXR writes them; the
// first line of the file is the image's top row (ImageIO.cpp:299-308).
int write_exr(const std::string& path, const float* pixels, uint32_t w, uint32_t h,
              uint32_t channels, bool half) {
    int r = check_image_args(path, pixels, w, h, channels);
    if (r) return r;
    // channel list in alphabetical order, each with its index in a pixel
    struct Ch { const char* name; uint32_t src; };
    static const Ch kY[1] = {{"Y", 0}};
    static const Ch kRgb[3] = {{"B", 2}, {"G", 1}, {"R", 0}};
    static const Ch kRgba[4] = {{"A", 3}, {"B", 2}, {"G", 1}, {"R", 0}};
    const Ch* chBegin = channels == 1 ? kY : (channels == 3 ? kRgb : kRgba);
    const size_t chCount = channels == 1 ? 1 : channels;
    struct Span {
        const Ch* b; size_t n;
        const Ch* begin() const { return b; }
        const Ch* end() const { return b + n; }
        size_t size() const { return n; }
    } chs{chBegin, chCount};
    const int32_t ptype = half ? 1 : 2;
    const uint32_t bpc = half ? 2 : 4;
    std::vector<uint8_t> b;
    append(b, int32_t(20000630));
    append(b, int32_t(2));
    attr_head(b, "channels", "chlist", int32_t(chs.size() * (2 + 16) + 1));
    for (const Ch& c : chs) {
        append_str(b, c.name);
        append(b, ptype);
        append(b, uint8_t(1));  // pLinear
        append(b, uint8_t(0));
        append(b, uint8_t(0));
        append(b, uint8_t(0));
        append(b, int32_t(1));  // x sampling
        append(b, int32_t(1));  // y sampling
    }
    append(b, uint8_t(0));
    attr_head(b, "compression", "compression", 1);
    append(b, uint8_t(0));
    const int32_t win[4] = {0, 0, int32_t(w) - 1, int32_t(h) - 1};
    attr_head(b, "dataWindow", "box2i", 16);
    for (int32_t v : win) append(b, v);
    attr_head(b, "displayWindow", "box2i", 16);
    for (int32_t v : win) append(b, v);
    attr_head(b, "lineOrder", "lineOrder", 1);
    append(b, uint8_t(0));
    attr_head(b, "pixelAspectRatio", "float", 4);
    append(b, 1.0f);
    attr_head(b, "screenWindowCenter", "v2f", 8);
    append(b, 0.0f);
    append(b, 0.0f);
    attr_head(b, "screenWindowWidth", "float", 4);
    append(b, 1.0f);
    append(b, uint8_t(0));  // end of header
    const size_t lineBytes = size_t(w) * chs.size() * bpc;
    const size_t table = b.size();
    b.resize(table + size_t(h) * 8);
    for (uint32_t y = 0; y < h; y++) {
        const uint64_t at = b.size();
        std::memcpy(b.data() + table + size_t(y) * 8, &at, 8);
        append(b, int32_t(y));
        append(b, int32_t(lineBytes));
        const uint32_t row = h - 1 - y;  // file line y = image row h-1-y
        for (const Ch& c : chs)
            for (uint32_t x = 0; x < w; x++) {
                const float v = pixels[(size_t(row) * w + x) * channels + c.src];
                if (half) append(b, f2h(v));
                else append(b, v);
            }
    }
    File out(path, "wb");
    if (!out.f) return io_error(path, "cannot open for writing");
    if (std::fwrite(b.data(), 1, b.size(), out.f) != b.size()) return io_error(path, "short write");
    return 0;
}

int read_exr(const std::string& path, std::vector<float>& pixels, uint32_t& w, uint32_t& h,
             uint32_t& channels) {
    std::vector<uint8_t> b;
    if (!read_all(path, b)) return io_error(path, "cannot read");
    size_t p = 0;
    auto need = [&](size_t n) { return b.size() - p >= n; };
    auto cstr = [&](std::string& s) {
        s.clear();
        while (p < b.size() && b[p]) s.push_back(static_cast<char>(b[p++]));
        if (p >= b.size()) return false;
        p++;
        return true;
    };
    int32_t magic = 0, version = 0;
    if (!need(8)) return io_error(path, "not an OpenEXR file");
    std::memcpy(&magic, b.data(), 4);
    std::memcpy(&version, b.data() + 4, 4);
    p = 8;
    if (magic != 20000630) return io_error(path, "not an OpenEXR file");
    if ((version & 0xFF) != 2 || (version & ~0x4FF))
        return io_error(path, "only single-part scanline OpenEXR files are read");
    struct Ch { std::string name; int32_t type; };
    std::vector<Ch> chs;
    int32_t win[4] = {0, 0, -1, -1};
    int compression = -1;
    bool haveWin = false;
    for (;;) {
        std::string name, type;
        if (!cstr(name)) return io_error(path, "truncated header");
        if (name.empty()) break;
        int32_t size = 0;
        if (!cstr(type) || !need(4)) return io_error(path, "truncated header");
        std::memcpy(&size, b.data() + p, 4);
        p += 4;
        if (size < 0 || !need(size_t(size))) return io_error(path, "truncated attribute");
        const size_t end = p + size_t(size);
        if (name == "channels" && type == "chlist") {
            while (p < end && b[p]) {
                Ch c;
                if (!cstr(c.name) || end - p < 16) return io_error(path, "bad channel list");
                std::memcpy(&c.type, b.data() + p, 4);
                int32_t xs, ys;
                std::memcpy(&xs, b.data() + p + 8, 4);
                std::memcpy(&ys, b.data() + p + 12, 4);
                if (xs != 1 || ys != 1 || c.type < 0 || c.type > 2)
                    return io_error(path, "subsampled or unknown channel type");
                p += 16;
                chs.push_back(c);
            }
        } else if (name == "compression" && size == 1) {
            compression = b[p];
        } else if (name == "dataWindow" && size == 16) {
            std::memcpy(win, b.data() + p, 16);
            haveWin = true;
        }
        p = end;
    }
    if (compression != 0) return io_error(path, "only NO_COMPRESSION OpenEXR files are read");
    if (!haveWin || chs.empty()) return io_error(path, "missing channels or data window");
    const int64_t W = int64_t(win[2]) - win[0] + 1, H = int64_t(win[3]) - win[1] + 1;
    if (W <= 0 || H <= 0 || W * H > (int64_t(1) << 30)) return io_error(path, "bad data window");
    // output layout: RGBA / RGB from R, G, B (, A), or the single channel
    int slot[4] = {-1, -1, -1, -1};
    for (size_t i = 0; i < chs.size(); i++) {
        const std::string& n = chs[i].name;
        if (n == "R") slot[0] = int(i);
        else if (n == "G") slot[1] = int(i);
        else if (n == "B") slot[2] = int(i);
        else if (n == "A") slot[3] = int(i);
    }
    const bool rgb = slot[0] >= 0 && slot[1] >= 0 && slot[2] >= 0;
    channels = rgb ? (slot[3] >= 0 ? 4u : 3u) : 1u;
    if (!rgb) slot[0] = 0;
    w = static_cast<uint32_t>(W);
    h = static_cast<uint32_t>(H);
    std::vector<size_t> chOff(chs.size());
    size_t lineBytes = 0;
    for (size_t i = 0; i < chs.size(); i++) {
        chOff[i] = lineBytes;
        lineBytes += size_t(W) * (chs[i].type == 1 ? 2 : 4);
    }
    if (!need(size_t(H) * 8)) return io_error(path, "truncated offset table");
    const size_t table = p;
    pixels.assign(size_t(W) * H * channels, 0.0f);
    for (int64_t k = 0; k < H; k++) {
        uint64_t at;
        std::memcpy(&at, b.data() + table + size_t(k) * 8, 8);
        if (at > b.size() || b.size() - at < 8 + lineBytes) return io_error(path, "bad line offset");
        int32_t y, size;
        std::memcpy(&y, b.data() + at, 4);
        std::memcpy(&size, b.data() + at + 4, 4);
        if (size_t(size) != lineBytes || y < win[1] || y > win[3])
            return io_error(path, "bad line block");
        const uint8_t* line = b.data() + at + 8;
        const size_t row = size_t(H - 1 - (int64_t(y) - win[1]));  // back to bottom-up rows
        for (uint32_t c = 0; c < channels; c++) {
            const size_t i = size_t(slot[c]);
            for (int64_t x = 0; x < W; x++) {
                float v;
                if (chs[i].type == 1) {
                    uint16_t hv;
                    std::memcpy(&hv, line + chOff[i] + size_t(x) * 2, 2);
                    v = h2f(hv);
                } else if (chs[i].type == 2) {
                    std::memcpy(&v, line + chOff[i] + size_t(x) * 4, 4);
                } else {
                    uint32_t u;
                    std::memcpy(&u, line + chOff[i] + size_t(x) * 4, 4);
                    v = static_cast<float>(u);
                }
                pixels[(row * size_t(W) + size_t(x)) * channels + c] = v;
            }
        }
    }
    return 0;
}

}  // namespace mrb

namespace mrb {
bool ends_with(const std::string& s, const char* suffix) {
    const size_t n = std::strlen(suffix);
    if (s.size() < n) return false;
    for (size_t i = 0; i < n; i++)
        if (std::tolower(static_cast<unsigned char>(s[s.size() - n + i])) != suffix[i]) return false;
    return true;
}

// Pixels divided by their sample counts (0 where the count is 0), written by
// extension: .exr (FLOAT) or .pfm.
int write_averaged(const std::string& p, const float* sums, const float* counts,
                   uint32_t countStride, uint32_t width, uint32_t height, uint32_t channels,
                   uint32_t outChannels) {
    if (!sums || !counts || !width || !height || channels == 0 || channels > 4 ||
        outChannels == 0 || outChannels > channels)
        return MRB_E_ARG;
    const size_t n = size_t(width) * height;
    std::vector<float> px(n * outChannels);
    for (size_t i = 0; i < n; i++) {
        const float w = counts[i * countStride];
        for (uint32_t c = 0; c < outChannels; c++)
            px[i * outChannels + c] = w != 0.0f ? sums[i * channels + c] / w : 0.0f;
    }
    if (ends_with(p, ".exr")) return write_exr(p, px.data(), width, height, outChannels, false);
    if (ends_with(p, ".pfm")) return write_pfm(p, px.data(), width, height, outChannels);
    set_error("%s: image files are .exr or .pfm", p.c_str());
    return MRB_E_UNSUPPORTED;
}
}  // namespace mrb

extern "C" {

int mrb_write_exr(const char* path, const float* pixels, uint32_t width, uint32_t height,
                  uint32_t channels, int half) {
    if (!path) return MRB_E_ARG;
    return mrb::write_exr(path, pixels, width, height, channels, half != 0);
}

int mrb_write_pfm(const char* path, const float* pixels, uint32_t width, uint32_t height,
                  uint32_t channels) {
    if (!path) return MRB_E_ARG;
    return mrb::write_pfm(path, pixels, width, height, channels);
}

int mrb_read_image(const char* path, float* pixels, size_t capacity, uint32_t* width,
                   uint32_t* height, uint32_t* channels) {
    if (!path || !width || !height || !channels) return MRB_E_ARG;
    std::vector<float> px;
    uint32_t w = 0, h = 0, c = 0;
    const std::string p(path);
    int r;
    if (mrb::ends_with(p, ".exr")) r = mrb::read_exr(p, px, w, h, c);
    else if (mrb::ends_with(p, ".pfm")) r = mrb::read_pfm(p, px, w, h, c);
    else {
        mrb::set_error("%s: image files are .exr or .pfm", path);
        return MRB_E_UNSUPPORTED;
    }
    if (r) return r;
    *width = w;
    *height = h;
    *channels = c;
    if (!pixels) return 0;
    if (capacity < px.size()) {
        mrb::set_error("%s: %zu floats needed, %zu given", path, px.size(), capacity);
        return MRB_E_ARG;
    }
    std::memcpy(pixels, px.data(), px.size() * 4);
    return 0;
}

}  // extern "C"
