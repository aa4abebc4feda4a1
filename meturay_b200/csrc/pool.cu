// Wavefront pool: continuous batching of render jobs on one device.
//
// Jobs (scene, camera, resolution, samples per frame, frame count, options)
// are submitted at any time.  A job is admitted when its image fits into
// the pool's HBM budget; admitted jobs share every iteration of the pool:
// one frame of each (as many as the wavefront's sample capacity holds,
// round robin) is generated, traced, partitioned and shaded in the same
// launches, and each job's frame is resolved into its own image.  A job is
// done after its frame count.  Jobs that arrive while others are on the
// GPU join at the next iteration.
//
// One iteration is one captured CUDA graph: the job table is copied from a
// pinned host buffer inside the graph, and every kernel reads its counts
// from the device, so the same graph serves any mix of jobs.
#include <algorithm>
#include <cstring>
#include <deque>
#include <memory>
#include <vector>

#include "objects.cuh"
#include "pool.cuh"
#include "shade.cuh"
#include "sort.cuh"

namespace {

using namespace mrb;

struct PoolJob {
    uint64_t id = 0;
    mrb_scene* scene = nullptr;
    CameraDev cam{};
    uint32_t width = 0, height = 0, samples = 1, frames = 1;
    uint32_t maxDepth = 5, rrStart = 3, nee = 1, mis = 0;
    uint64_t seed = 1;
    uint32_t framesDone = 0;
    uint32_t state = 0;  // MRB_JOB_QUEUED / ACTIVE / DONE
    size_t bytes = 0;    // HBM the job holds while admitted (its image)
    DBuf image;
    uint32_t sampleCount() const { return width * samples * height * samples; }
};

}  // namespace

struct mrb_pool {
    mrb_system* sys = nullptr;
    cudaStream_t stream = nullptr;
    uint32_t capacity = 0;   // camera samples per iteration
    uint32_t maxDepth = 5;   // depths per iteration (the deepest job's)
    uint32_t idBits = 1;
    int block = 128, stack = 128;
    size_t budget = 0, used = 0;
    uint32_t maxRays = 0;
    DBuf rayO[2], rayD[2], aux[2], count, hitKey, hitPrim, hitT, hitBary, dense, sortedIds,
        portion, samplesBuf, counters, errorFlags, sortTemp, table;
    size_t sortTempBytes = 0;
    unsigned char* hostTable = nullptr;  // pinned: PoolHeader + JobDev[kPoolMaxJobs]
    std::vector<std::unique_ptr<PoolJob>> jobs;
    std::deque<PoolJob*> queue;
    std::vector<PoolJob*> active;
    uint64_t nextId = 1;
    size_t rr = 0;
    uint64_t iterations = 0;
    cudaGraphExec_t graph = nullptr;
    bool graphDirty = true;
    // Image buffers of released jobs, kept for the next admissions: a
    // cudaMalloc per admission and a cudaFree (which waits for the whole
    // device) per release cost milliseconds each inside the serving loop.
    // Bounded by kSpareBytes, and freed (oldest first) before a new buffer
    // would take the admitted and kept images past the HBM budget.
    std::vector<std::pair<void*, size_t>> spare;
    size_t spareBytes = 0;
    // pinned staging for image read-back
    void* stage = nullptr;
    size_t stageBytes = 0;
    ~mrb_pool() {
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamSynchronize(stream);
        if (hostTable) cudaFreeHost(hostTable);
        if (stage) cudaFreeHost(stage);
        for (auto& b : spare) cudaFree(b.first);
        if (stream) cudaStreamDestroy(stream);
    }
    static constexpr size_t kSpareBytes = size_t(1) << 30;
    // a kept buffer of at least `bytes` and at most 4x that, else a new one
    int take_image(DBuf& img, size_t bytes) {
        int best = -1;
        for (size_t i = 0; i < spare.size(); i++)
            if (spare[i].second >= bytes && spare[i].second <= 4 * bytes &&
                (best < 0 || spare[i].second < spare[size_t(best)].second))
                best = int(i);
        if (best < 0) {
            // a new buffer: kept ones go first where they would take the
            // images past the budget
            while (!spare.empty() && used + spareBytes + bytes > budget) {
                cudaFree(spare.front().first);
                spareBytes -= spare.front().second;
                spare.erase(spare.begin());
            }
            return img.alloc(bytes);
        }
        img.release();
        img.p = spare[size_t(best)].first;
        img.bytes = spare[size_t(best)].second;
        spareBytes -= img.bytes;
        spare.erase(spare.begin() + best);
        return 0;
    }
    void keep_image(DBuf& img) {
        if (!img.p) return;
        spare.emplace_back(img.p, img.bytes);
        spareBytes += img.bytes;
        img.p = nullptr;
        img.bytes = 0;
        while (spareBytes > kSpareBytes && !spare.empty()) {
            cudaFree(spare.front().first);
            spareBytes -= spare.front().second;
            spare.erase(spare.begin());
        }
    }
    PoolHeader* header() { return reinterpret_cast<PoolHeader*>(hostTable); }
    JobDev* hostJobs() { return reinterpret_cast<JobDev*>(hostTable + sizeof(PoolHeader)); }
    const PoolHeader* devHeader() const { return table.as<PoolHeader>(); }
    const JobDev* devJobs() const {
        return reinterpret_cast<const JobDev*>(table.as<unsigned char>() + sizeof(PoolHeader));
    }
    PoolJob* find(uint64_t id) {
        for (auto& j : jobs)
            if (j && j->id == id) return j.get();
        return nullptr;
    }
};

namespace {

constexpr size_t kTableBytes = sizeof(PoolHeader) + sizeof(JobDev) * kPoolMaxJobs;

int pool_buffers(mrb_pool* p) {
    const uint32_t maxRays = 2 * p->capacity;
    p->maxRays = maxRays;
    int r;
    for (int i = 0; i < 2; i++) {
        if ((r = p->rayO[i].alloc(size_t(maxRays) * 16)) || (r = p->rayD[i].alloc(size_t(maxRays) * 16)) ||
            (r = p->aux[i].alloc(size_t(maxRays) * sizeof(RayAux))))
            return r;
    }
    if ((r = p->count.alloc(8)) || (r = p->hitKey.alloc(size_t(maxRays) * 4)) ||
        (r = p->hitPrim.alloc(size_t(maxRays) * 4)) || (r = p->hitT.alloc(size_t(maxRays) * 4)) ||
        (r = p->hitBary.alloc(size_t(maxRays) * 8)) || (r = p->dense.alloc(size_t(maxRays) * 4)) ||
        (r = p->sortedIds.alloc(size_t(maxRays) * 4)) || (r = p->portion.alloc(32 * 4)) ||
        (r = p->samplesBuf.alloc(size_t(p->capacity) * 16)) || (r = p->counters.alloc(16)) ||
        (r = p->errorFlags.alloc(16)) || (r = p->table.alloc(kTableBytes)))
        return r;
    p->sortTempBytes = radix_sort_temp_bytes(maxRays, 4, 0, 3 + 24);
    if ((r = p->sortTemp.alloc(p->sortTempBytes))) return r;
    MRB_CUDA(cudaMemsetAsync(p->counters.p, 0, 16, p->stream));
    MRB_CUDA(cudaMemsetAsync(p->errorFlags.p, 0, 16, p->stream));
    return 0;
}

size_t pool_fixed_bytes(uint32_t capacity) {
    const size_t R = 2 * size_t(capacity);
    return 2 * R * (16 + 16 + sizeof(RayAux)) + R * (4 + 4 + 4 + 8 + 4 + 4) + size_t(capacity) * 16 +
           radix_sort_temp_bytes(static_cast<uint32_t>(R), 4, 0, 3 + 24) + kTableBytes;
}

// One iteration: camera rays of every selected job, maxDepth depths of
// trace / partition / shade, then each job's resolve.
int record_iteration(mrb_pool* p) {
    int r;
    cudaStream_t st = p->stream;
    uint32_t* cnt = p->count.as<uint32_t>();
    MRB_CUDA(cudaMemcpyAsync(p->table.p, p->hostTable, kTableBytes, cudaMemcpyHostToDevice, st));
    if ((r = pool_camera(p->devHeader(), p->devJobs(), p->capacity, p->rayO[0].as<float4>(),
                         p->rayD[0].as<float4>(), p->aux[0].as<RayAux>(),
                         p->samplesBuf.as<float4>(), cnt, st)))
        return r;
    uint32_t* port = p->portion.as<uint32_t>();
    const PortionTable pt{port, port + 8, port + 16};
    for (uint32_t d = 0; d < p->maxDepth; d++) {
        const int cur = d & 1, nxt = cur ^ 1;
        const HitOut ho{p->hitKey.as<uint32_t>(), p->hitPrim.as<uint32_t>(), p->hitT.as<float>(),
                        p->hitBary.as<float2>()};
        if ((r = trace_closest_wide_jobs(p->devJobs(), p->aux[cur].as<RayAux>(),
                                         p->rayO[cur].as<float4>(), p->rayD[cur].as<float4>(),
                                         cnt + cur, p->maxRays, ho,
                                         p->errorFlags.as<uint32_t>(), p->block, p->stack, st)))
            return r;
        // also adds this wavefront to the traced-ray total and clears the
        // next wavefront's counter
        if ((r = dense_keys(ho.key, cnt + cur, p->maxRays, p->idBits, p->dense.as<uint32_t>(), pt,
                            st, p->counters.as<unsigned long long>(), cnt + nxt)))
            return r;
        if ((r = radix_sort_pairs<uint32_t>(p->dense.as<uint32_t>(), p->sortedIds.as<uint32_t>(),
                                            cnt + cur, p->maxRays, 0, 3 + int(p->idBits), true,
                                            p->sortTemp.p, p->sortTempBytes, st, true)))
            return r;
        if ((r = find_portions(p->dense.as<uint32_t>(), cnt + cur, p->maxRays, p->idBits, pt, st)))
            return r;
        const HitIn hi{ho.key, ho.prim, ho.t, ho.bary};
        if ((r = shade_jobs(p->devJobs(), p->rayO[cur].as<float4>(), p->rayD[cur].as<float4>(),
                            p->aux[cur].as<RayAux>(), hi, p->sortedIds.as<uint32_t>(), pt.nonNull,
                            p->maxRays, p->samplesBuf.as<float4>(), p->rayO[nxt].as<float4>(),
                            p->rayD[nxt].as<float4>(), p->aux[nxt].as<RayAux>(), cnt + nxt, st)))
            return r;
    }
    return pool_resolve(p->devHeader(), p->devJobs(), p->capacity, p->samplesBuf.as<float4>(), st);
}

int pool_graph(mrb_pool* p) {
    if (!p->graphDirty && p->graph) return 0;
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    // an empty table first, so one-time kernel setup runs outside the capture
    PoolHeader* h = p->header();
    const PoolHeader keep = *h;
    *h = PoolHeader{0, 0, 0, 0};
    int r = record_iteration(p);
    MRB_CUDA(cudaStreamSynchronize(p->stream));
    *h = keep;
    if (r) return r;
    cudaGraph_t g = nullptr;
    MRB_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    r = record_iteration(p);
    cudaError_t e = cudaStreamEndCapture(p->stream, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) {
        set_error("pool: graph capture failed: %s", cudaGetErrorString(e));
        return MRB_E_CUDA;
    }
    e = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        set_error("pool: graph instantiate failed: %s", cudaGetErrorString(e));
        return MRB_E_CUDA;
    }
    p->graphDirty = false;
    return 0;
}

JobDev job_dev(const PoolJob& j) {
    JobDev d{};
    d.sc = j.scene->dev();
    d.wide = j.scene->wide();
    d.cam = j.cam;
    d.image = j.image.as<float4>();
    d.width = j.width;
    d.height = j.height;
    d.samples = j.samples;
    d.maxDepth = j.maxDepth;
    d.rrStart = j.rrStart;
    d.nee = j.nee;
    d.mis = j.mis;
    d.seedLo = static_cast<uint32_t>(j.seed);
    d.seedHi = static_cast<uint32_t>(j.seed >> 32);
    d.frame = j.framesDone;
    d.sampleCount = j.sampleCount();
    return d;
}

}  // namespace

extern "C" {

int mrb_pool_create(mrb_system* sys, uint32_t capacity, uint32_t max_depth, size_t hbm_budget,
                    mrb_pool** out) {
    if (!sys || !out || capacity == 0 || capacity > (1u << 28) || max_depth == 0 ||
        max_depth > 255) {
        mrb::set_error("pool: capacity must be in [1, 2^28] samples and max depth in [1, 255]");
        return MRB_E_ARG;
    }
    *out = nullptr;
    MRB_CUDA(cudaSetDevice(sys->device));
    auto p = std::make_unique<mrb_pool>();
    p->sys = sys;
    p->capacity = capacity;
    p->maxDepth = max_depth;
    MRB_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    MRB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&p->hostTable), kTableBytes,
                           cudaHostAllocDefault));
    std::memset(p->hostTable, 0, kTableBytes);
    // the admission budget: what the caller grants, else the free memory now
    // minus the pool's own buffers and a 10 % reserve
    size_t freeB = 0, totalB = 0;
    MRB_CUDA(cudaMemGetInfo(&freeB, &totalB));
    const size_t fixed = pool_fixed_bytes(capacity);
    if (hbm_budget == 0) {
        const size_t reserve = totalB / 10;
        hbm_budget = freeB > fixed + reserve ? freeB - fixed - reserve : 0;
    }
    p->budget = hbm_budget;
    int r = pool_buffers(p.get());
    if (r) return r;
    MRB_CUDA(cudaStreamSynchronize(p->stream));
    *out = p.release();
    return 0;
}

void mrb_pool_destroy(mrb_pool* p) { delete p; }

int mrb_pool_set_launch(mrb_pool* p, int trace_block, int trace_stack) {
    if (!p || (trace_block != 64 && trace_block != 128 && trace_block != 256) ||
        (trace_stack != 0 && trace_stack != 64 && trace_stack != 128)) {
        mrb::set_error("pool: traversal block 64/128/256 and stack 64/128 (or 0: octant order)");
        return MRB_E_ARG;
    }
    p->block = trace_block;
    p->stack = trace_stack;
    p->graphDirty = true;
    return 0;
}

int mrb_pool_submit(mrb_pool* p, mrb_scene* scene, const mrb_pool_job* desc, uint64_t* job_id) {
    if (!p || !scene || !desc || !job_id) return MRB_E_ARG;
    if (!scene->built || scene->T == 0 || (scene->T > 1 && !scene->wNodes.p)) {
        mrb::set_error("pool: the scene's accelerator is not built");
        return MRB_E_STATE;
    }
    auto j = std::make_unique<PoolJob>();
    j->scene = scene;
    j->width = desc->width;
    j->height = desc->height;
    j->samples = desc->samples ? desc->samples : 1;
    j->frames = desc->frames ? desc->frames : 1;
    j->maxDepth = desc->max_depth;
    j->rrStart = desc->rr_start;
    j->nee = desc->nee ? 1 : 0;
    j->mis = desc->mis ? 1 : 0;
    j->seed = desc->seed;
    if (j->width == 0 || j->height == 0 || j->samples > 64 || j->maxDepth == 0 ||
        j->maxDepth > p->maxDepth) {
        mrb::set_error("pool: job needs a size, samples <= 64 and max depth in [1, %u]",
                       p->maxDepth);
        return MRB_E_ARG;
    }
    if (uint64_t(j->width) * j->samples * j->height * j->samples > p->capacity) {
        mrb::set_error("pool: one frame of the job (%ux%u, %u^2 spp) exceeds the wavefront "
                       "capacity of %u samples",
                       j->width, j->height, j->samples, p->capacity);
        return MRB_E_ARG;
    }
    j->bytes = size_t(j->width) * j->height * 16;
    if (j->bytes > p->budget) {
        mrb::set_error("pool: the job's image (%zu bytes) exceeds the HBM budget (%zu)", j->bytes,
                       p->budget);
        return MRB_E_OOM;
    }
    float f[14];
    mrb_camera_frame(&desc->camera, f);
    for (int i = 0; i < 3; i++) {
        j->cam.position[i] = f[i];
        j->cam.bottomLeft[i] = f[3 + i];
        j->cam.right[i] = f[6 + i];
        j->cam.up[i] = f[9 + i];
    }
    j->cam.planeSize[0] = f[12];
    j->cam.planeSize[1] = f[13];
    j->cam.nearFar[0] = desc->camera.near_far[0];
    j->cam.nearFar[1] = desc->camera.near_far[1];
    j->id = p->nextId++;
    j->state = MRB_JOB_QUEUED;
    if (scene->idBits > p->idBits) {
        p->idBits = scene->idBits;
        p->graphDirty = true;
    }
    *job_id = j->id;
    p->queue.push_back(j.get());
    p->jobs.push_back(std::move(j));
    return 0;
}

int mrb_pool_step(mrb_pool* p, uint32_t* finished, uint32_t* active, uint32_t* queued) {
    if (!p) return MRB_E_ARG;
    MRB_CUDA(cudaSetDevice(p->sys->device));
    // admission, first come first served, while the images fit the budget
    while (!p->queue.empty() && p->used + p->queue.front()->bytes <= p->budget &&
           p->active.size() < kPoolMaxJobs) {
        PoolJob* j = p->queue.front();
        int r = p->take_image(j->image, j->bytes);
        if (r) {
            // the budget was optimistic: wait until memory frees up
            if (p->active.empty()) return r;
            break;
        }
        MRB_CUDA(cudaMemsetAsync(j->image.p, 0, j->bytes, p->stream));
        p->used += j->bytes;
        j->state = MRB_JOB_ACTIVE;
        p->active.push_back(j);
        p->queue.pop_front();
    }
    uint32_t done = 0;
    if (!p->active.empty()) {
        // this iteration's jobs: round robin from rr while the wavefront holds them
        std::vector<PoolJob*> sel;
        uint32_t samples = 0, pixels = 0;
        JobDev* tab = p->hostJobs();
        const size_t A = p->active.size();
        for (size_t k = 0; k < A && sel.size() < kPoolMaxJobs; k++) {
            PoolJob* j = p->active[(p->rr + k) % A];
            const uint32_t n = j->sampleCount();
            if (samples + n > p->capacity) continue;
            JobDev d = job_dev(*j);
            d.sampleBase = samples;
            d.pixelBase = pixels;
            tab[sel.size()] = d;
            sel.push_back(j);
            samples += n;
            pixels += j->width * j->height;
        }
        *p->header() = PoolHeader{static_cast<uint32_t>(sel.size()), samples, pixels, 0};
        int r = pool_graph(p);
        if (r) return r;
        MRB_CUDA(cudaGraphLaunch(p->graph, p->stream));
        MRB_CUDA(cudaStreamSynchronize(p->stream));
        uint32_t e[2] = {0, 0};
        MRB_CUDA(cudaMemcpy(e, p->errorFlags.p, 4, cudaMemcpyDeviceToHost));
        MRB_CUDA(cudaMemcpy(e + 1, radix_sort_error_flag(p->sortTemp.p, p->maxRays), 4,
                            cudaMemcpyDeviceToHost));
        if (e[0] || e[1]) {
            mrb::set_error("pool: device-side limit hit (trace flag %u, sort flag %u)", e[0], e[1]);
            return MRB_E_DEVICE;
        }
        p->iterations++;
        p->rr = (p->rr + sel.size()) % A;
        for (PoolJob* j : sel) {
            j->framesDone++;
            if (j->framesDone >= j->frames) {
                j->state = MRB_JOB_DONE;
                done++;
            }
        }
        p->active.erase(std::remove_if(p->active.begin(), p->active.end(),
                                       [](PoolJob* j) { return j->state == MRB_JOB_DONE; }),
                        p->active.end());
    }
    if (finished) *finished = done;
    if (active) *active = static_cast<uint32_t>(p->active.size());
    if (queued) *queued = static_cast<uint32_t>(p->queue.size());
    return 0;
}

int mrb_pool_job_status(mrb_pool* p, uint64_t id, uint32_t* state, uint32_t* frames_done) {
    if (!p) return MRB_E_ARG;
    PoolJob* j = p->find(id);
    if (!j) {
        mrb::set_error("pool: no job %llu", static_cast<unsigned long long>(id));
        return MRB_E_ARG;
    }
    if (state) *state = j->state;
    if (frames_done) *frames_done = j->framesDone;
    return 0;
}

int mrb_pool_job_image(mrb_pool* p, uint64_t id, float* host_rgba, int release) {
    if (!p) return MRB_E_ARG;
    PoolJob* j = p->find(id);
    if (!j || j->state != MRB_JOB_DONE) {
        mrb::set_error("pool: job %llu is not done", static_cast<unsigned long long>(id));
        return MRB_E_STATE;
    }
    if (host_rgba) {
        if (!j->image.p) {
            mrb::set_error("pool: job %llu's image was released", static_cast<unsigned long long>(id));
            return MRB_E_STATE;
        }
        // through pinned staging on the pool's stream
        if (p->stageBytes < j->bytes) {
            if (p->stage) cudaFreeHost(p->stage);
            p->stage = nullptr;
            p->stageBytes = 0;
            MRB_CUDA(cudaHostAlloc(&p->stage, j->bytes, cudaHostAllocDefault));
            p->stageBytes = j->bytes;
        }
        MRB_CUDA(cudaMemcpyAsync(p->stage, j->image.p, j->bytes, cudaMemcpyDeviceToHost, p->stream));
        MRB_CUDA(cudaStreamSynchronize(p->stream));
        std::memcpy(host_rgba, p->stage, j->bytes);
    }
    if (release && j->image.p) {
        p->keep_image(j->image);
        p->used -= j->bytes;
        for (auto& u : p->jobs)
            if (u.get() == j) u.reset();
    }
    return 0;
}

int mrb_pool_stats(mrb_pool* p, uint64_t* rays, uint64_t* iterations, size_t* hbm_used,
                   size_t* hbm_budget) {
    if (!p) return MRB_E_ARG;
    if (rays) {
        unsigned long long r = 0;
        MRB_CUDA(cudaMemcpy(&r, p->counters.p, 8, cudaMemcpyDeviceToHost));
        *rays = r;
    }
    if (iterations) *iterations = p->iterations;
    if (hbm_used) *hbm_used = p->used;
    if (hbm_budget) *hbm_budget = p->budget;
    return 0;
}

void* mrb_pool_stream(mrb_pool* p) { return p ? static_cast<void*>(p->stream) : nullptr; }

}  // extern "C"
