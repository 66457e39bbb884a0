// Render server: batched / continuous multi-request path tracing over resident scenes.
//
// Two path pools of P slots that alternate between iterations: an iteration's live paths
// occupy slots [0, live) of its pool, new camera paths are appended after them, and
// shading moves each continuing path to the next free slot of the other pool, so every
// stage reads path state in nearly slot order.  Each pool iteration (one CUDA graph
// launch):
//   k_plan      issues min(free slots, unissued tickets) tickets; resets this
//               iteration's queue counters (single thread)
//   k_generate  turns tickets into camera paths: ticket t -> (request, pixel, sample)
//               through the admitted requests' ticket ranges (binary search)
//   k_extend    closest hits of every queued path (mixed depths, requests and scenes)
//               by persistent warps with refilling lanes; misses retire
//   k_shade     per-material shading (the same per-path code as lux_render)
//   k_shadow    NEE shadow rays (persistent warps with refilling lanes)
//   k_retire    finished paths add their radiance to their request's film in 64-bit
//               fixed point (order-independent) and count towards completion
// Tickets enumerate each request's paths pixel-major (pixel = idx / spp), so the random
// numbers of a path depend only on (request seed, pixel, sample): a request renders the
// same whether alone or mixed.  The host worker thread admits requests by memory budget,
// uploads request slots and ticket ranges between launches (stream order), keeps two
// iterations in flight, and delivers films when a request's retired-path count reaches
// its path count.
// No reference counterpart: the reference renders one request per call with a host
// loop over batches and bounces (integrator/wavefront_scheduler.cu:73-131).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lux_gpu.h"
#include "pt_kernels.cuh"
#include "pt_scene.h"

namespace lux {
namespace pt {
namespace {

constexpr int kMaxRequests = 1024;
constexpr float kFixedScale = 4294967296.0f;  // 2^32
constexpr float kFixedMax = 1e9f;             // per-sample clamp keeps 64-bit sums exact

struct ReqSlot {
    int scene, width, height, spp, max_depth, light_sampler, cancelled, pad;
    uint64_t seed;
    int frame_index, sample_offset;
    long long ticket_start, total;
    unsigned long long* film;
};

struct TicketMap {
    int count;
    int pad;
    long long start[kMaxRequests];
    int slot[kMaxRequests];
};

struct ServerState {
    int live;          // live paths in this iteration's pool, slots [0, live)
    int live_next;     // continuing paths appended to the other pool
    int gen_count;     // tickets issued this iteration
    int gen_live;      // of which started paths (slots live + [0, gen_live))
    long long gen_ticket;
    long long next_ticket;
    long long ticket_limit;
    int count_ray[2];
    int count_mat[kClasses];
    int count_shadow;
    int count_term;
    int extend_next;   // refill cursor of k_extend_s
    int shadow_next;   // refill cursor of k_shadow_s
    int pad2;
    unsigned long long rays[2];
};

struct ServerDev {
    PathPool pool[2];  // path state alternates between the two; queues, hit and shadow
                       // records are shared (pool[1] aliases pool[0]'s)
    int* req_of[2];    // request slot of each path, per pool
    int* sh_dest;      // where a shadow ray's path now lives: 2 * slot + (1: other pool)
    int* qterm;
    ServerState* st;
    const ReqSlot* req;
    const TicketMap* tmap;
    const SceneView* scenes;
    int scene_count;
    unsigned long long* done;
    int* error;
};

constexpr int kMaxScenes = 64;
static_assert(sizeof(SceneView) % 4 == 0, "scene views are staged as words");

// Each kernel first copies the scene table into shared memory (dynamic, scene_count
// views), so per-path and per-step scene reads are shared-memory reads rather than
// dependent global loads.
extern __shared__ __align__(16) unsigned char g_stage[];

LUX_D const SceneView* stage_scenes(const ServerDev& d) {
    SceneView* dst = reinterpret_cast<SceneView*>(g_stage);
    const int words = d.scene_count * static_cast<int>(sizeof(SceneView) / 4);
    const int* src = reinterpret_cast<const int*>(d.scenes);
    int* out = reinterpret_cast<int*>(dst);
    for (int i = threadIdx.x; i < words; i += blockDim.x) out[i] = src[i];
    __syncthreads();
    return dst;
}

LUX_HD size_t scene_stage_bytes(int scene_count) { return sizeof(SceneView) * static_cast<size_t>(scene_count); }

__global__ void k_plan(ServerState* st, int capacity) {
    const int live = st->live_next;  // the previous iteration's continuing paths
    st->live = live;
    st->live_next = 0;
    long long avail = st->ticket_limit - st->next_ticket;
    if (avail < 0) avail = 0;
    const int n = static_cast<int>(min(static_cast<long long>(capacity - live), avail));
    st->gen_count = n;
    st->gen_live = 0;
    st->gen_ticket = st->next_ticket;
    st->next_ticket += n;
    for (int k = 0; k < kClasses; ++k) st->count_mat[k] = 0;
    st->count_shadow = 0;
    st->count_term = 0;
    st->extend_next = 0;
    st->shadow_next = 0;
}

// Ticket t of request q is its path idx = t - ticket_start, sample-major: pixel
// idx % (width * height), sample idx / (width * height).  Consecutive tickets are
// neighbouring pixels, and one pixel's samples are a frame apart, so retiring paths
// rarely meet on the same film words.
__global__ void __launch_bounds__(kThreads) k_generate(ServerDev d, int cur) {
    const SceneView* scenes = stage_scenes(d);
    // The ticket map follows the scene table in shared memory.
    const int tcount = min(d.tmap->count, kMaxRequests);
    long long* tstart = reinterpret_cast<long long*>(g_stage + scene_stage_bytes(d.scene_count));
    int* tslot = reinterpret_cast<int*>(tstart + kMaxRequests);
    for (int k = threadIdx.x; k < tcount; k += blockDim.x) {
        tstart[k] = d.tmap->start[k];
        tslot[k] = d.tmap->slot[k];
    }
    __syncthreads();
    const int n = d.st->gen_count;
    const int live = d.st->live;
    const long long t0 = d.st->gen_ticket;
    const PathPool& pool = d.pool[cur];
    const int stride = gridDim.x * blockDim.x;
    const int rounds = (n + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        const int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        const bool active = i < n;
        bool dead = false;
        int rs = -1;
        long long idx = 0;
        if (active && tcount <= 0) {  // cannot happen: tickets imply a request
            atomicOr(d.error, kErrLoopBound);
        } else if (active) {
            const long long t = t0 + i;
            int lo = 0, hi = tcount - 1;
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (tstart[mid] <= t) lo = mid;
                else hi = mid - 1;
            }
            rs = tslot[lo];
            const ReqSlot& q = d.req[rs];
            idx = t - q.ticket_start;
            if (q.cancelled || idx < 0 || idx >= q.total || q.scene < 0 ||
                q.scene >= d.scene_count) {
                if (!q.cancelled) atomicOr(d.error, kErrLoopBound);
                dead = true;  // counts towards completion, contributes nothing
            }
        }
        const bool start = active && rs >= 0 && !dead;
        const int slot = append(&d.st->gen_live, 0, start);
        if (start) {
            const ReqSlot& q = d.req[rs];
            const long long npix = static_cast<long long>(q.width) * q.height;
            init_path(pool, scenes[q.scene].camera, live + slot, static_cast<int>(idx % npix),
                      static_cast<int>(idx / npix),
                      CameraParams{q.width, q.height, q.seed, q.frame_index, q.sample_offset});
            d.req_of[cur][live + slot] = rs;
        }
        // Tickets of cancelled requests are done at once (one atomic per warp and request).
        const bool skip = active && rs >= 0 && dead;
        const unsigned mask = __ballot_sync(0xffffffffu, skip);
        if (skip) {
            const unsigned peers = __match_any_sync(mask, rs);
            if (static_cast<int>(threadIdx.x & 31) == __ffs(peers) - 1)
                atomicAdd(d.done + rs, static_cast<unsigned long long>(__popc(peers)));
        }
    }
}

// The bounce kernels run at three resident blocks per SM (at most 80 registers, small
// spills) rather than the two their register counts allow: config 4 went from 684 to
// 812 Mrays/s on one B200.
__global__ void __launch_bounds__(kThreads, 3) k_extend_s(ServerDev d, int cur, int budget) {
    const SceneView* scenes = stage_scenes(d);
    const int n = d.st->live + d.st->gen_live;  // slots [0, n) of this iteration's pool
    const PathPool& pool = d.pool[cur];
    const int* req_of = d.req_of[cur];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&d.st->rays[0], static_cast<unsigned long long>(n));
    refill_walks(
        pool, nullptr, n, &d.st->extend_next, budget, d.error,
        [&](int p) { return req_of[p]; },
        [&](int rs) -> const SceneView& { return scenes[d.req[rs].scene]; },
        [&](int p, int rs, const SceneHit& h) {
            int cls = -1;
            if (p >= 0) {
                const ReqSlot& q = d.req[rs];
                cls = extend_finish(pool, scenes[q.scene], q.light_sampler, p, h);
            }
            const bool hit = cls >= 0;
            const int slot = append(d.st->count_mat, hit ? cls : 0, hit);
            if (hit) pool.qmat[cls * pool.capacity + slot] = p;
            const int qt = append(&d.st->count_term, 0, p >= 0 && !hit);
            if (qt >= 0) d.qterm[qt] = p;
        });
}

// Shading in place; a path that continues moves to the other pool at the next
// appended slot, so the next iteration reads its paths in slot order.
__global__ void __launch_bounds__(kThreads, 3) k_shade_s(ServerDev d, int cur) {
    const SceneView* scenes = stage_scenes(d);
    const int nxt = cur ^ 1;
    const PathPool& pool = d.pool[cur];
    int c[kClasses];
    int total = 0;
    for (int k = 0; k < kClasses; ++k) {
        c[k] = d.st->count_mat[k];
        total += c[k];
    }
    const int stride = gridDim.x * blockDim.x;
    const int rounds = (total + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        const int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        const bool active = i < total;
        int cls = 0, j = i;
        while (cls < kClasses - 1 && j >= c[cls]) j -= c[cls++];
        const int p = active ? pool.qmat[cls * pool.capacity + j] : 0;
        const int rs = active ? d.req_of[cur][p] : 0;
        ShadeOut o;
        if (active) {
            const ReqSlot& q = d.req[rs];
            o = shade_path(pool, scenes[q.scene], q.light_sampler, q.max_depth, p);
        }
        const int s = append(&d.st->count_shadow, 0, o.shadow);
        if (o.shadow) pool.qshadow[s] = p;
        const int q = append(&d.st->live_next, 0, o.spawn);
        if (o.spawn) {
            copy_path(pool, p, d.pool[nxt], q);
            d.req_of[nxt][q] = rs;
        }
        if (active) d.sh_dest[p] = o.spawn ? 2 * q + 1 : 2 * p;
        const int t = append(&d.st->count_term, 0, active && !o.spawn);
        if (t >= 0) d.qterm[t] = p;
    }
}

__global__ void __launch_bounds__(kThreads, 3) k_shadow_s(ServerDev d, int cur, int budget) {
    const SceneView* scenes = stage_scenes(d);
    const PathPool& pool = d.pool[cur];
    const int* req_of = d.req_of[cur];
    unsigned long long segments = 0;
    refill_shadows(
        pool, pool.qshadow, d.st->count_shadow, &d.st->shadow_next, budget, d.error,
        [&](int p) { return req_of[p]; },
        [&](int rs) -> const SceneView& { return scenes[d.req[rs].scene]; },
        [&](int p, f3 v) {
            const int dest = d.sh_dest[p];
            add_radiance(d.pool[cur ^ (dest & 1)], dest >> 1, v);
        },
        segments);
    warp_add(&d.st->rays[1], segments);
}

LUX_D unsigned long long to_fixed(float v) {
    v = fminf(fmaxf(v, 0.0f), kFixedMax);  // NaN -> 0
    return static_cast<unsigned long long>(__float2ll_rn(v * kFixedScale));
}

__global__ void __launch_bounds__(kThreads) k_retire(ServerDev d, int cur) {
    const PathPool& pool = d.pool[cur];
    const int n = d.st->count_term;
    const int stride = gridDim.x * blockDim.x;
    const int rounds = (n + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        int i = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool active = i < n;
        int p = active ? d.qterm[i] : 0;
        int rs = active ? d.req_of[cur][p] : -1;
        if (active) {
            const ReqSlot& q = d.req[rs];
            int pixel = pool.meta[p].x;
            if (!q.cancelled && pixel >= 0 && pixel < q.width * q.height) {
                float4 rad = pool.rad[p];
                unsigned long long* f = q.film + 3 * static_cast<size_t>(pixel);
                atomicAdd(f, to_fixed(rad.x));
                atomicAdd(f + 1, to_fixed(rad.y));
                atomicAdd(f + 2, to_fixed(rad.z));
            }
        }
        // completion counts: one atomic per (warp, request)
        unsigned mask = __ballot_sync(0xffffffffu, active);
        if (active) {
            unsigned peers = __match_any_sync(mask, rs);
            if (static_cast<int>(threadIdx.x & 31) == __ffs(peers) - 1)
                atomicAdd(d.done + rs, static_cast<unsigned long long>(__popc(peers)));
        }
    }
}

__global__ void k_fixed_to_float(const unsigned long long* film, float* out, size_t n) {
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = __ll2float_rn(static_cast<long long>(film[i])) * (1.0f / kFixedScale);
}

int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace pt
}  // namespace lux

struct lux_server_request {
    int64_t id = 0;
    int scene = 0;
    lux_render_request req{};
    float* out = nullptr;
    bool out_device = false;
    int state = LUX_REQ_QUEUED;
    int slot = -1;
    long long ticket_start = 0, total = 0;
    unsigned long long* film = nullptr;
    float* staging = nullptr;
    size_t bytes = 0;
    int64_t t_submit = 0, t_admit = 0, t_done = 0;
    int64_t admit_iter = 0;   // first pool iteration launched after the admission
    bool cancel_requested = false;
    cudaEvent_t delivered = nullptr;
};

struct lux_server {
    lux_ctx* ctx = nullptr;
    std::vector<lux_scene*> scenes;
    lux::pt::SceneView* d_scenes = nullptr;
    lux::pt::PathPool pool[2];      // pool[1] owns only its path-state arrays
    int* req_of[2] = {nullptr, nullptr};
    int* sh_dest = nullptr;
    int* qterm = nullptr;
    lux::pt::ServerState* st = nullptr;
    lux::pt::ReqSlot* d_req = nullptr;
    lux::pt::ReqSlot* h_req = nullptr;         // pinned mirror
    lux::pt::TicketMap* d_tmap = nullptr;
    lux::pt::TicketMap* h_tmap = nullptr;      // pinned mirror
    unsigned long long* d_done = nullptr;
    unsigned long long* h_done[2] = {nullptr, nullptr};  // pinned, per in-flight iteration
    lux::pt::ServerState* h_state[2] = {nullptr, nullptr};
    long long* h_limit = nullptr;              // pinned ticket limit
    cudaEvent_t iter_done[2] = {nullptr, nullptr};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // Request films come from this pool, which keeps freed memory (release threshold at
    // its maximum): the default pool returns memory to the driver at every stream
    // synchronisation and maps it again on the next allocation, which stalled the worker
    // for hundreds of milliseconds.
    cudaMemPool_t film_pool = nullptr;
    int max_requests = 256;
    int64_t budget = 0;
    int64_t used = 0;
    int64_t pool_bytes = 0;
    long long ticket_limit = 0;
    // host state
    std::mutex mu;
    std::condition_variable wake;
    std::condition_variable finished;
    std::deque<int64_t> pending;
    std::map<int64_t, std::unique_ptr<lux_server_request>> requests;
    std::vector<int> free_slots;
    std::vector<int64_t> active;               // admitted, in ticket order
    std::vector<int64_t> delivering;
    struct MeshUpdate {
        int scene, mesh;
        std::vector<float> vertices;
    };
    std::deque<MeshUpdate> updates;
    int64_t next_id = 1;
    int64_t launched = 0;    // pool iterations launched
    int64_t collected = 0;   // iterations whose counters were read back
    bool stop = false;
    int64_t iterations = 0, completed = 0, admitted = 0, refits = 0;
    int64_t longest_pass_ns = 0;      // longest worker loop pass (admission latency bound)
    int64_t longest_wait_ns = 0;      // longest wait for one iteration's counters
    unsigned long long rays[2] = {0, 0};
    int error_status = 0;
    std::thread worker;
};

namespace {

using lux::pt::ReqSlot;

int server_fail(int st, const std::string& m) { return lux::fail(st, m); }

int64_t request_cost(const lux_server_request& r) {
    int64_t pixels = static_cast<int64_t>(r.req.width) * r.req.height;
    return pixels * 3 * 8 + (r.out_device ? 0 : pixels * 3 * 4);
}

void upload_tmap(lux_server* s) {
    s->h_tmap->count = 0;
    for (int64_t id : s->active) {
        auto& r = *s->requests[id];
        int k = s->h_tmap->count++;
        s->h_tmap->start[k] = r.ticket_start;
        s->h_tmap->slot[k] = r.slot;
    }
    size_t bytes = offsetof(lux::pt::TicketMap, start) + sizeof(long long) * lux::pt::kMaxRequests
                 + sizeof(int) * lux::pt::kMaxRequests;
    cudaMemcpyAsync(s->d_tmap, s->h_tmap, bytes, cudaMemcpyHostToDevice, s->ctx->stream);
}

// Admits queued requests in order while slots and budget allow.  Called with mu held.
void admit(lux_server* s) {
    bool changed = false;
    while (!s->pending.empty() && !s->free_slots.empty()) {
        auto& r = *s->requests[s->pending.front()];
        int64_t cost = request_cost(r);
        if (s->used + cost > s->budget) break;
        cudaStream_t stream = s->ctx->stream;
        size_t n = static_cast<size_t>(r.req.width) * r.req.height * 3;
        if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.film), n * 8, s->film_pool,
                                    stream) != cudaSuccess) {
            cudaGetLastError();
            break;
        }
        if (!r.out_device &&
            cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.staging), n * 4, s->film_pool,
                                    stream) != cudaSuccess) {
            cudaGetLastError();
            cudaFreeAsync(r.film, stream);
            r.film = nullptr;
            break;
        }
        cudaMemsetAsync(r.film, 0, n * 8, stream);
        r.slot = s->free_slots.back();
        s->free_slots.pop_back();
        r.bytes = cost;
        s->used += cost;
        r.total = static_cast<long long>(r.req.width) * r.req.height * r.req.spp;
        r.ticket_start = s->ticket_limit;
        s->ticket_limit += r.total;
        ReqSlot q{};
        q.scene = r.scene;
        q.width = r.req.width;
        q.height = r.req.height;
        q.spp = r.req.spp;
        q.max_depth = r.req.max_depth;
        q.light_sampler = r.req.light_sampler;
        q.cancelled = 0;
        q.seed = r.req.seed;
        q.frame_index = r.req.frame_index;
        q.sample_offset = r.req.sample_offset;
        q.ticket_start = r.ticket_start;
        q.total = r.total;
        q.film = r.film;
        s->h_req[r.slot] = q;
        cudaMemcpyAsync(s->d_req + r.slot, s->h_req + r.slot, sizeof(ReqSlot),
                        cudaMemcpyHostToDevice, stream);
        cudaMemsetAsync(s->d_done + r.slot, 0, sizeof(unsigned long long), stream);
        r.state = LUX_REQ_RUNNING;
        r.t_admit = lux::pt::now_ns();
        r.admit_iter = s->launched;
        s->active.push_back(r.id);
        s->pending.pop_front();
        ++s->admitted;
        changed = true;
    }
    if (changed) {
        upload_tmap(s);
        *s->h_limit = s->ticket_limit;
        cudaMemcpyAsync(&s->st->ticket_limit, s->h_limit, sizeof(long long),
                        cudaMemcpyHostToDevice, s->ctx->stream);
    }
}

// Finishes requests whose retired-path count reached their path count.  done: the
// counters read back after pool iteration `iter` (-1: none); a request admitted after
// that iteration was launched is not judged by them (its slot may still show the
// previous occupant's count).  mu held.
void collect(lux_server* s, const unsigned long long* done, int64_t iter) {
    bool changed = false;
    cudaStream_t stream = s->ctx->stream;
    for (size_t k = 0; k < s->active.size();) {
        auto& r = *s->requests[s->active[k]];
        if (!done || iter < r.admit_iter || static_cast<long long>(done[r.slot]) < r.total) {
            ++k;
            continue;
        }
        size_t n = static_cast<size_t>(r.req.width) * r.req.height * 3;
        if (!r.cancel_requested) {
            float* dst = r.out_device ? r.out : r.staging;
            int grid = std::max(1, std::min(s->ctx->sm_count * 4, static_cast<int>((n + 255) / 256)));
            lux::pt::k_fixed_to_float<<<grid, 256, 0, stream>>>(r.film, dst, n);
            if (!r.out_device)
                cudaMemcpyAsync(r.out, r.staging, n * 4, cudaMemcpyDeviceToHost, stream);
        }
        cudaFreeAsync(r.film, stream);
        if (r.staging) cudaFreeAsync(r.staging, stream);
        r.film = nullptr;
        r.staging = nullptr;
        cudaEventCreateWithFlags(&r.delivered, cudaEventDisableTiming);
        cudaEventRecord(r.delivered, stream);
        s->free_slots.push_back(r.slot);
        s->used -= r.bytes;
        s->delivering.push_back(r.id);
        s->active.erase(s->active.begin() + k);
        changed = true;
    }
    if (changed) upload_tmap(s);
    for (size_t k = 0; k < s->delivering.size();) {
        auto& r = *s->requests[s->delivering[k]];
        if (cudaEventQuery(r.delivered) != cudaSuccess) {
            cudaGetLastError();
            ++k;
            continue;
        }
        cudaEventDestroy(r.delivered);
        r.delivered = nullptr;
        r.state = r.cancel_requested ? LUX_REQ_CANCELLED : LUX_REQ_DONE;
        r.t_done = lux::pt::now_ns();
        ++s->completed;
        s->delivering.erase(s->delivering.begin() + k);
        s->finished.notify_all();
    }
}

void fail_all(lux_server* s, int status) {
    s->error_status = status;
    for (auto& kv : s->requests) {
        auto& r = *kv.second;
        if (r.state == LUX_REQ_QUEUED || r.state == LUX_REQ_RUNNING) r.state = LUX_REQ_FAILED;
    }
    s->pending.clear();
    s->active.clear();
    s->finished.notify_all();
}

void worker_main(lux_server* s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    int64_t pass_start = lux::pt::now_ns();
    for (;;) {
        {
            const int64_t t = lux::pt::now_ns();
            s->longest_pass_ns = std::max(s->longest_pass_ns, t - pass_start);
            pass_start = t;
        }
        if (s->stop) break;
        if (s->error_status == 0) admit(s);
        if (!s->updates.empty()) {
            // One batch of vertex updates per iteration, the latest per mesh; updates that
            // arrive while it is applied wait for the next iteration, so a producer faster
            // than the refits cannot starve the render.
            std::deque<lux_server::MeshUpdate> batch;
            batch.swap(s->updates);
            lk.unlock();
            int64_t applied = 0;
            for (size_t k = 0; k < batch.size(); ++k) {
                bool superseded = false;
                for (size_t j = k + 1; j < batch.size() && !superseded; ++j)
                    superseded = batch[j].scene == batch[k].scene && batch[j].mesh == batch[k].mesh;
                if (superseded) continue;
                lux_scene* scene = s->scenes[batch[k].scene];
                bool view_changed = false;
                if (lux::scene_update_mesh(s->ctx, scene, batch[k].mesh,
                                           batch[k].vertices.data(), false,
                                           &view_changed) != LUX_OK)
                    continue;
                ++applied;
                // Re-derived light tables: the staged view follows, in stream order before
                // the next iteration.  (A copy from pageable memory may wait for the
                // stream, so it is made only when the view changed.)
                if (view_changed)
                    cudaMemcpyAsync(s->d_scenes + batch[k].scene, &scene->view,
                                    sizeof(scene->view), cudaMemcpyHostToDevice, s->ctx->stream);
            }
            lk.lock();
            s->refits += applied;
        }
        bool busy = !s->active.empty() || !s->delivering.empty();
        if (!busy && s->launched == s->collected) {
            s->wake.wait(lk, [&] {
                return s->stop || (!s->pending.empty() && !s->free_slots.empty()) ||
                       !s->updates.empty();
            });
            pass_start = lux::pt::now_ns();  // idling is not a stall
            continue;
        }
        // Keep up to two iterations in flight: launch one, then read the older one's
        // counters while the newer runs.
        bool launch = !s->active.empty() && s->launched - s->collected < 2;
        cudaEvent_t delivering_event = s->delivering.empty()
                                           ? nullptr
                                           : s->requests[s->delivering.front()]->delivered;
        int64_t launch_index = s->launched;
        if (launch) ++s->launched;
        lk.unlock();
        if (launch) {
            int parity = static_cast<int>(launch_index & 1);
            cudaGraphLaunch(s->graph[parity], s->ctx->stream);
            cudaMemcpyAsync(s->h_done[parity], s->d_done,
                            sizeof(unsigned long long) * s->max_requests, cudaMemcpyDeviceToHost,
                            s->ctx->stream);
            cudaMemcpyAsync(s->h_state[parity], s->st, sizeof(lux::pt::ServerState),
                            cudaMemcpyDeviceToHost, s->ctx->stream);
            cudaEventRecord(s->iter_done[parity], s->ctx->stream);
        }
        int err_word = 0;
        int64_t read_iter = -1;
        int64_t wait_ns = 0;
        if (s->collected < s->launched) {
            read_iter = s->collected;
            const int64_t w0 = lux::pt::now_ns();
            cudaError_t e = cudaEventSynchronize(s->iter_done[static_cast<int>(read_iter & 1)]);
            wait_ns = lux::pt::now_ns() - w0;
            if (e != cudaSuccess) {
                lk.lock();
                fail_all(s, LUX_ERR_CUDA);
                continue;
            }
            cudaMemcpy(&err_word, s->ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost);
        } else if (delivering_event) {
            cudaEventSynchronize(delivering_event);  // the oldest film delivery
        }
        lk.lock();
        s->longest_wait_ns = std::max(s->longest_wait_ns, wait_ns);
        if (read_iter >= 0) {
            int parity = static_cast<int>(read_iter & 1);
            s->collected = read_iter + 1;
            ++s->iterations;
            s->rays[0] = s->h_state[parity]->rays[0];
            s->rays[1] = s->h_state[parity]->rays[1];
            if (err_word) {
                cudaMemset(s->ctx->d_error, 0, sizeof(int));
                fail_all(s, LUX_ERR_DEVICE_CHECK);
                continue;
            }
            collect(s, s->h_done[parity], read_iter);
        } else {
            collect(s, nullptr, -1);
        }
    }
}

int build_graphs(lux_server* s) {
    using namespace lux::pt;
    ServerDev d;
    for (int k = 0; k < 2; ++k) {
        d.pool[k] = s->pool[k];
        d.req_of[k] = s->req_of[k];
    }
    d.sh_dest = s->sh_dest;
    d.qterm = s->qterm;
    d.st = s->st;
    d.req = s->d_req;
    d.tmap = s->d_tmap;
    d.scenes = s->d_scenes;
    d.scene_count = static_cast<int>(s->scenes.size());
    d.done = s->d_done;
    d.error = s->ctx->d_error;
    const size_t stage = scene_stage_bytes(d.scene_count);
    const size_t gen_stage = stage + (sizeof(long long) + sizeof(int)) * kMaxRequests;
    cudaFuncSetAttribute(k_generate, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(gen_stage));
    int grid = s->ctx->sm_count * 8;
    int extend_blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&extend_blocks, k_extend_s, kThreads, stage);
    const int extend_grid = s->ctx->sm_count * std::max(extend_blocks, 1);
    int shadow_blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shadow_blocks, k_shadow_s, kThreads, stage);
    const int shadow_grid = s->ctx->sm_count * std::max(shadow_blocks, 1);
    cudaStream_t stream = s->ctx->stream;
    for (int cur = 0; cur < 2; ++cur) {
        cudaGraph_t g;
        cudaError_t err = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (err != cudaSuccess) return lux::cuda_fail(err, "graph capture");
        k_plan<<<1, 1, 0, stream>>>(s->st, s->pool[0].capacity);
        k_generate<<<grid, kThreads, gen_stage, stream>>>(d, cur);
        k_extend_s<<<extend_grid, kThreads, stage, stream>>>(d, cur, s->ctx->path_budget);
        k_shade_s<<<grid, kThreads, stage, stream>>>(d, cur);
        k_shadow_s<<<shadow_grid, kThreads, stage, stream>>>(d, cur, s->ctx->path_budget);
        k_retire<<<grid, kThreads, 0, stream>>>(d, cur);
        err = cudaStreamEndCapture(stream, &g);
        if (err != cudaSuccess) return lux::cuda_fail(err, "graph capture end");
        err = cudaGraphInstantiate(&s->graph[cur], g, 0);
        cudaGraphDestroy(g);
        if (err != cudaSuccess) return lux::cuda_fail(err, "graph instantiate");
    }
    return LUX_OK;
}

void server_release(lux_server* s) {
    if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
    for (int k = 0; k < 2; ++k) {
        if (s->graph[k]) cudaGraphExecDestroy(s->graph[k]);
        if (s->iter_done[k]) cudaEventDestroy(s->iter_done[k]);
        if (s->h_done[k]) cudaFreeHost(s->h_done[k]);
        if (s->h_state[k]) cudaFreeHost(s->h_state[k]);
    }
    lux::pt::path_pool_free(s->pool[0]);
    const lux::pt::PathPool& p1 = s->pool[1];
    void* dev[] = {s->d_scenes, s->req_of[0], s->req_of[1], s->sh_dest, s->qterm, s->st,
                   s->d_req, s->d_tmap, s->d_done, p1.thr_eta, p1.rad, p1.prev, p1.meta,
                   p1.rng, p1.ray_o, p1.ray_d};
    for (void* p : dev)
        if (p) cudaFree(p);
    if (s->h_req) cudaFreeHost(s->h_req);
    if (s->h_tmap) cudaFreeHost(s->h_tmap);
    if (s->h_limit) cudaFreeHost(s->h_limit);
    for (auto& kv : s->requests) {
        cudaStream_t stream = s->ctx ? s->ctx->stream : nullptr;
        if (kv.second->film) cudaFreeAsync(kv.second->film, stream);
        if (kv.second->staging) cudaFreeAsync(kv.second->staging, stream);
        if (kv.second->delivered) cudaEventDestroy(kv.second->delivered);
    }
    if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
    if (s->film_pool) cudaMemPoolDestroy(s->film_pool);
    if (s->ctx) lux_ctx_destroy(s->ctx);
}

}  // namespace

extern "C" {

int lux_server_create(int device, lux_scene* const* scenes, int32_t scene_count,
                      const lux_server_options* options, lux_server** out) {
    using namespace lux::pt;
    if (!out || (scene_count > 0 && !scenes) || scene_count <= 0)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "server needs at least one scene");
    *out = nullptr;
    lux_server_options opt{};
    if (options) opt = *options;
    int64_t pool_paths = opt.pool_paths > 0 ? opt.pool_paths : (1 << 22);
    if (pool_paths > (1 << 28)) return server_fail(LUX_ERR_INVALID_ARGUMENT, "pool too large");
    int max_requests = opt.max_requests > 0 ? opt.max_requests : 256;
    if (max_requests > kMaxRequests)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "max_requests above 1024");
    if (scene_count > lux::pt::kMaxScenes)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "a server holds at most 64 resident scenes");
    for (int i = 0; i < scene_count; ++i)
        if (!scenes[i]) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null scene");
    auto* s = new (std::nothrow) lux_server();
    if (!s) return server_fail(LUX_ERR_OUT_OF_MEMORY, "server allocation failed");
    int st = lux_ctx_create(&s->ctx, device, nullptr);
    if (st) {
        delete s;
        return st;
    }
    if (opt.path_budget > 0) s->ctx->path_budget = std::min(opt.path_budget, 4096);
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&s->film_pool, &props) == cudaSuccess) {
            uint64_t keep = ~uint64_t(0);
            cudaMemPoolSetAttribute(s->film_pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            cudaGetLastError();
            s->film_pool = nullptr;
            st = server_fail(LUX_ERR_CUDA, "film memory pool");
        }
    }
    s->scenes.assign(scenes, scenes + scene_count);
    s->max_requests = max_requests;
    s->budget = opt.memory_budget_bytes > 0 ? opt.memory_budget_bytes : (int64_t(120) << 30);
    int cap = static_cast<int>(pool_paths);
    st = path_pool_alloc(s->pool[0], cap);
    std::vector<SceneView> views;
    for (lux_scene* sc : s->scenes) views.push_back(sc->view);
    auto dmalloc = [&](void** p, size_t bytes) {
        if (st) return;
        if (cudaMalloc(p, bytes) != cudaSuccess) {
            cudaGetLastError();
            st = server_fail(LUX_ERR_OUT_OF_MEMORY, "server allocation failed");
        }
    };
    dmalloc(reinterpret_cast<void**>(&s->d_scenes), sizeof(SceneView) * views.size());
    // The second pool: its own path state, the first pool's queues and records.
    if (!st) {
        PathPool& p1 = s->pool[1];
        p1 = s->pool[0];
        p1.thr_eta = p1.rad = p1.prev = p1.ray_o = p1.ray_d = nullptr;
        p1.meta = nullptr;
        p1.rng = nullptr;
    }
    for (float4** a : {&s->pool[1].thr_eta, &s->pool[1].rad, &s->pool[1].prev, &s->pool[1].ray_o,
                       &s->pool[1].ray_d})
        dmalloc(reinterpret_cast<void**>(a), sizeof(float4) * cap);
    dmalloc(reinterpret_cast<void**>(&s->pool[1].meta), sizeof(int4) * cap);
    dmalloc(reinterpret_cast<void**>(&s->pool[1].rng), sizeof(uint4) * cap);
    dmalloc(reinterpret_cast<void**>(&s->req_of[0]), sizeof(int) * cap);
    dmalloc(reinterpret_cast<void**>(&s->req_of[1]), sizeof(int) * cap);
    dmalloc(reinterpret_cast<void**>(&s->sh_dest), sizeof(int) * cap);
    dmalloc(reinterpret_cast<void**>(&s->qterm), sizeof(int) * cap);
    dmalloc(reinterpret_cast<void**>(&s->st), sizeof(ServerState));
    dmalloc(reinterpret_cast<void**>(&s->d_req), sizeof(ReqSlot) * max_requests);
    dmalloc(reinterpret_cast<void**>(&s->d_tmap), sizeof(TicketMap));
    dmalloc(reinterpret_cast<void**>(&s->d_done), sizeof(unsigned long long) * max_requests);
    auto hmalloc = [&](void** p, size_t bytes) {
        if (st) return;
        if (cudaMallocHost(p, bytes) != cudaSuccess) {
            cudaGetLastError();
            st = server_fail(LUX_ERR_OUT_OF_MEMORY, "pinned allocation failed");
        }
    };
    hmalloc(reinterpret_cast<void**>(&s->h_req), sizeof(ReqSlot) * max_requests);
    hmalloc(reinterpret_cast<void**>(&s->h_tmap), sizeof(TicketMap));
    hmalloc(reinterpret_cast<void**>(&s->h_limit), sizeof(long long));
    for (int k = 0; k < 2; ++k) {
        hmalloc(reinterpret_cast<void**>(&s->h_done[k]), sizeof(unsigned long long) * max_requests);
        hmalloc(reinterpret_cast<void**>(&s->h_state[k]), sizeof(ServerState));
        if (!st) cudaEventCreateWithFlags(&s->iter_done[k], cudaEventDisableTiming);
    }
    if (!st) {
        cudaStream_t stream = s->ctx->stream;
        cudaMemcpyAsync(s->d_scenes, views.data(), sizeof(SceneView) * views.size(),
                        cudaMemcpyHostToDevice, stream);
        ServerState init{};  // no live paths
        cudaMemcpyAsync(s->st, &init, sizeof(init), cudaMemcpyHostToDevice, stream);
        cudaMemsetAsync(s->d_done, 0, sizeof(unsigned long long) * max_requests, stream);
        std::memset(s->h_tmap, 0, sizeof(TicketMap));
        std::memset(s->h_done[0], 0, sizeof(unsigned long long) * max_requests);
        std::memset(s->h_done[1], 0, sizeof(unsigned long long) * max_requests);
        cudaMemcpyAsync(s->d_tmap, s->h_tmap, sizeof(TicketMap), cudaMemcpyHostToDevice, stream);
        st = lux::cuda_fail(cudaStreamSynchronize(stream), "server init");
    }
    if (!st) st = build_graphs(s);
    if (st) {
        server_release(s);
        delete s;
        return st;
    }
    // Pool, queues and records, plus the second pool's path state and request slots.
    s->pool_bytes = static_cast<int64_t>(cap) * (16 * 12 + 4 * 7 + 4 * kClasses + 16 * 7 + 4 + 4);
    s->used = s->pool_bytes;
    for (int k = max_requests - 1; k >= 0; --k) s->free_slots.push_back(k);
    s->worker = std::thread(worker_main, s);
    *out = s;
    return LUX_OK;
}

int lux_server_submit(lux_server* s, int32_t scene, const lux_render_request* req,
                      float* film_sum, int64_t* request_id) {
    if (!s || !req || !film_sum || !request_id)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (scene < 0 || scene >= static_cast<int>(s->scenes.size()))
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "scene index out of range");
    if (req->width <= 0 || req->height <= 0 || req->spp <= 0)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "render requires a non-empty film");
    if (req->max_depth < 0 || req->max_depth > 1000)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "max_depth must be in 0..1000");
    if (req->light_sampler < 0 || req->light_sampler > 2)
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "light sampler: 0 uniform, 1 power or 2 tree");
    if (static_cast<long long>(req->width) * req->height > (1ll << 30))
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "image too large");
    auto r = std::make_unique<lux_server_request>();
    r->scene = scene;
    r->req = *req;
    r->out = film_sum;
    r->out_device = lux::pt::is_device_ptr(film_sum);
    r->t_submit = lux::pt::now_ns();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error_status) return server_fail(s->error_status, "server failed earlier");
    if (s->pool_bytes + request_cost(*r) > s->budget)
        return server_fail(LUX_ERR_BUDGET, "request film does not fit the memory budget");
    r->id = s->next_id++;
    *request_id = r->id;
    s->pending.push_back(r->id);
    s->requests[r->id] = std::move(r);
    s->wake.notify_all();
    return LUX_OK;
}

int lux_server_poll(lux_server* s, int64_t id, int32_t* state) {
    if (!s || !state) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return server_fail(LUX_ERR_INVALID_ARGUMENT, "unknown request");
    *state = it->second->state;
    return LUX_OK;
}

static bool final_state(int st) {
    return st == LUX_REQ_DONE || st == LUX_REQ_CANCELLED || st == LUX_REQ_FAILED;
}

int lux_server_wait(lux_server* s, int64_t id, int64_t timeout_us, int32_t* state) {
    if (!s) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return server_fail(LUX_ERR_INVALID_ARGUMENT, "unknown request");
    lux_server_request* r = it->second.get();
    auto pred = [&] { return final_state(r->state); };
    if (timeout_us < 0) s->finished.wait(lk, pred);
    else s->finished.wait_for(lk, std::chrono::microseconds(timeout_us), pred);
    if (state) *state = r->state;
    return LUX_OK;
}

int lux_server_wait_all(lux_server* s, int64_t timeout_us) {
    if (!s) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] {
        for (auto& kv : s->requests)
            if (!final_state(kv.second->state)) return false;
        return true;
    };
    bool ok = timeout_us < 0 ? (s->finished.wait(lk, pred), true)
                             : s->finished.wait_for(lk, std::chrono::microseconds(timeout_us), pred);
    if (s->error_status) return server_fail(s->error_status, "server failed");
    return ok ? LUX_OK : server_fail(LUX_ERR_INVALID_ARGUMENT, "timed out");
}

int lux_server_cancel(lux_server* s, int64_t id) {
    if (!s) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return server_fail(LUX_ERR_INVALID_ARGUMENT, "unknown request");
    lux_server_request& r = *it->second;
    if (r.state == LUX_REQ_QUEUED) {
        s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), id), s->pending.end());
        r.state = LUX_REQ_CANCELLED;
        r.cancel_requested = true;
        s->finished.notify_all();
    } else if (r.state == LUX_REQ_RUNNING && !r.cancel_requested) {
        r.cancel_requested = true;
        s->h_req[r.slot].cancelled = 1;
        cudaMemcpyAsync(&s->d_req[r.slot].cancelled, &s->h_req[r.slot].cancelled, sizeof(int),
                        cudaMemcpyHostToDevice, s->ctx->stream);
    }
    return LUX_OK;
}

int lux_server_update_mesh(lux_server* s, int32_t scene, int32_t mesh, const float* vertices) {
    if (!s || !vertices) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    if (scene < 0 || scene >= static_cast<int>(s->scenes.size()))
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "scene index out of range");
    lux_scene* sc = s->scenes[scene];
    if (mesh < 0 || mesh >= static_cast<int>(sc->mesh_vertices.size()))
        return server_fail(LUX_ERR_INVALID_ARGUMENT, "mesh out of range");
    lux_server::MeshUpdate u{scene, mesh,
                             std::vector<float>(vertices, vertices + sc->mesh_vertices[mesh].size())};
    std::lock_guard<std::mutex> lk(s->mu);
    s->updates.push_back(std::move(u));
    s->wake.notify_all();
    return LUX_OK;
}

int lux_server_request_times(lux_server* s, int64_t id, int64_t* times) {
    if (!s || !times) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return server_fail(LUX_ERR_INVALID_ARGUMENT, "unknown request");
    times[0] = it->second->t_submit;
    times[1] = it->second->t_admit;
    times[2] = it->second->t_done;
    return LUX_OK;
}

int lux_server_stats(lux_server* s, int64_t* stats) {
    if (!s || !stats) return server_fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    stats[0] = s->iterations;
    stats[1] = static_cast<int64_t>(s->rays[0]);
    stats[2] = static_cast<int64_t>(s->rays[1]);
    stats[3] = s->completed;
    stats[4] = s->admitted;
    stats[5] = s->refits;
    stats[6] = s->used;
    stats[7] = s->longest_pass_ns;
    stats[8] = s->longest_wait_ns;
    return LUX_OK;
}

int lux_server_destroy(lux_server* s) {
    if (!s) return LUX_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->wake.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    server_release(s);
    delete s;
    return LUX_OK;
}

}  // extern "C"
