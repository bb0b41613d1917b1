// Request server: continuous batching of ray-trace jobs into persistent
// tracer kernels.
//
// Memory: one device arena of `budget_bytes` (a single cudaMalloc at
// create) holds the packed grids (an LRU cache keyed by the caller) and each
// admitted job's rays, sort workspace and outputs. A job is admitted, in
// arrival order, when its grid and its memory fit and a job-table slot is
// free; otherwise it waits. Idle grids (no admitted job) are evicted LRU to
// make room.
//
// Scheduling: each call of sloth_server_step() (1) retires iterations that
// have finished on the GPU, (2) admits waiting jobs: rays are copied into the
// arena, the grid is packed if it is not resident, the Morton pre-pass sorts
// the rays and the job's kernel arguments are written to its table slot, and
// (3) if an iteration slot is free, hands out 1024-ray tiles round-robin to
// all admitted jobs (`quantum` tiles per job per round, up to
// `tiles_per_step`) and launches the iteration: a captured CUDA graph that
// copies the work list to the device and runs one persistent serving kernel
// per tracer mode on parallel branches (the inverse-bremsstrahlung path times
// the interior fast path, each kernel with one copy of the step). Two iterations can be in flight on
// two streams, so one iteration's tail overlaps the next one's start. Jobs
// that arrive while others are running join at the next iteration and their
// tiles run in the same kernels as the others' (continuous batching).
//
// Each ray is traced by exactly the code of the single-trace kernel
// (trace_tile in tracer.cuh), so a job's results do not depend on which
// other jobs share its iterations.
#include <atomic>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <set>
#include <unordered_map>
#include <vector>

#include "tracer.cuh"

namespace sloth {

// Tracer modes: the inverse-bremsstrahlung path (IB_OFF, IB_SUBCRITICAL,
// IB_GENERAL) times the fast path (interior runs with interior sampling when
// the job's density range allows them, none otherwise); mode = 2 * IB + fast.
constexpr int kModes = 6;

struct WorkItem {
    int slot;
    int tile;
};

struct WorkHeader {
    int counter[kModes];   // tiles taken so far (zero when the iteration starts)
    int count[kModes];     // tiles of each mode
    int offset[kModes];    // first item of each mode
    int pad;
};

template <int IB, int FAST>
__global__ void __launch_bounds__(kThreads, SLOTH_TRACE_MIN_BLOCKS)
serve_kernel(const TraceArgs* __restrict__ table, WorkHeader* hdr, const WorkItem* __restrict__ items, int mode) {
    __shared__ TraceArgs s_args;
    __shared__ unsigned s_key[kTile];
    __shared__ unsigned s_id[kTile];
    __shared__ int s_item, s_slot, s_newslot, s_tile, s_head;
    __shared__ unsigned long long s_steps;
    CellCacheFor<PolF32, IB> cc;
    cc.base = 0xffffffffu;
    if (threadIdx.x == 0) {
        s_slot = -1;
        s_steps = 0;
    }
    const int count = hdr->count[mode];
    const int offset = hdr->offset[mode];
    for (;;) {
        if (threadIdx.x == 0) {
            const int w = atomicAdd(&hdr->counter[mode], 1);
            s_item = w;
            s_head = 0;
            if (w < count) {
                const WorkItem it = items[offset + w];
                s_tile = it.tile;
                s_newslot = it.slot;
            }
        }
        __syncthreads();
        if (s_item >= count) break;
        if (s_newslot != s_slot) {
            // a tile of another job: its arguments into shared memory, and
            // the cell cache no longer refers to the same grid
            const unsigned* src = reinterpret_cast<const unsigned*>(table + s_newslot);
            unsigned* dst = reinterpret_cast<unsigned*>(&s_args);
            for (int i = threadIdx.x; i < (int)(sizeof(TraceArgs) / 4); i += blockDim.x) dst[i] = src[i];
            cc.base = 0xffffffffu;
            __syncthreads();
            if (threadIdx.x == 0) s_slot = s_newslot;
        }
        const long long start = (long long)s_tile * kTile;
        const int cnt = (int)min((long long)kTile, s_args.n - start);
        unsigned long long my_steps = 0;
        // FAST: the job's density range bounds its accelerations (the host
        // sorted its tiles by interior_sampling_ok)
        trace_tile<PolF32, IB, FAST>(s_args, start, cnt, s_key, s_id, &s_head, cc, my_steps);
        block_add(my_steps, &s_steps, s_args.total_steps);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
class Arena {
  public:
    int init(size_t bytes, int* alloc_counter);
    void destroy() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
    }
    // first fit, 256-byte granules
    bool alloc(size_t bytes, size_t* off) {
        bytes = (bytes + 255u) & ~(size_t)255u;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes;
                const size_t at = it->first + bytes;
                free_.erase(it);
                if (rest) free_[at] = rest;
                used_ += bytes;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + 255u) & ~(size_t)255u;
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    char* ptr(size_t off) const { return base_ + off; }
    size_t size() const { return size_; }
    size_t used() const { return used_; }

  private:
    char* base_ = nullptr;
    size_t size_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;
};

struct GridEntry {
    uint64_t key;
    SlothGridDesc desc;
    double omega;
    size_t off = 0, bytes = 0;
    int refs = 0;
    unsigned long long last_use = 0;
};

enum JobState {
    JOB_PENDING = SLOTH_JOB_PENDING,
    JOB_ADMITTED = SLOTH_JOB_RUNNING,
    JOB_DONE = SLOTH_JOB_DONE,
    JOB_FETCHING = SLOTH_JOB_FETCHING,
    JOB_FETCHED = SLOTH_JOB_FETCHED,
};

struct Job {
    int id = -1;
    int state = JOB_PENDING;
    uint64_t grid_key = 0;
    SlothGridDesc desc{};
    const void* ne = nullptr;
    int ne_is_f64 = 0;
    SlothTraceParams p{};
    const float* rays_src = nullptr;
    int rays_on_host = 0;
    long long n = 0;
    // admitted
    int slot = -1;
    size_t off = 0, bytes = 0;
    int tiles_total = 0, tiles_assigned = 0;
    long long last_iter = -1;      // iteration that ran the job's last tiles
    int mode = 0;
    SlothTraceOutputs out{};       // device pointers in the arena
    cudaEvent_t fetched = nullptr;
};

// Memory of a cancelled RUNNING job, released once the iterations that
// hold its tiles have finished.
struct DeferredFree {
    size_t off = 0, bytes = 0;
    int slot = -1;
    uint64_t grid_key = 0;
    long long last_iter = -1;
};

struct IterSlot {
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t start = nullptr;    // timing events around the iteration's graph
    cudaEvent_t done = nullptr;
    WorkHeader* h_buf = nullptr;    // pinned: header + items
    WorkHeader* d_buf = nullptr;    // device copy
    long long iter = -1;            // iteration in flight, -1 when free
};

struct ServerImpl {
    SlothServerConfig cfg{};
    int device = 0;
    int sms = 148;
    Arena arena;
    TraceArgs* d_table = nullptr;
    TraceArgs* h_table = nullptr;   // pinned staging of the table rows
    std::vector<int> free_slots;
    std::unordered_map<uint64_t, GridEntry> grids;
    std::unordered_map<int, Job> jobs;
    std::deque<int> pending;
    std::vector<int> admitted;      // jobs holding a slot, in admission order
    std::vector<DeferredFree> deferred;   // cancelled running jobs' memory
    size_t rr = 0;                  // round-robin cursor into `admitted`
    int next_id = 1;
    unsigned long long clock = 0;
    long long iter_next = 0;
    long long iter_done = -1;          // every iteration <= iter_done has finished
    std::set<long long> finished;      // finished iterations above iter_done
    cudaEvent_t t0 = nullptr;          // time origin of the iteration intervals
    std::map<long long, std::pair<double, double>> intervals;   // finished, not yet merged (ms from t0)
    double busy_end = 0.0, first_start = -1.0;
    IterSlot it[2];
    cudaStream_t admit = nullptr;   // uploads, packing, pre-pass, table rows
    cudaStream_t copy = nullptr;    // result downloads
    cudaEvent_t admit_ev = nullptr;
    SlothServerStats stats{};
    std::mutex mu;
};

static size_t job_bytes(long long n, const SlothTraceParams* p, int* bbits_out, size_t* parts) {
    const size_t N = (size_t)(n > 0 ? n : 1);
    const size_t S = (size_t)p->n_saves;
    const int bbits = bucket_bits_for(n);
    if (bbits_out) *bbits_out = bbits;
    size_t sz[10];
    sz[0] = align256(6 * N * 4);                  // rays
    sz[1] = align256(S * 4 * N * 4);              // jones
    sz[2] = align256(S * N * 8);                  // phase
    sz[3] = align256(p->inv_brems ? S * N * 4 : 4);  // amp
    sz[4] = align256(N);                          // status
    sz[5] = align256(N * 4);                      // steps
    sz[6] = 256;                                  // total steps
    sz[7] = align256(((size_t)4 << bbits));       // histogram
    sz[8] = align256(N * 4) * 3;                  // keys, perm, sorted keys
    size_t total = 0;
    for (int i = 0; i < 9; ++i) {
        if (parts) parts[i] = total;
        total += sz[i];
    }
    return total;
}

static int graph_build(ServerImpl* s, IterSlot& is, int blocks[kModes]) {
    // captured once per iteration slot: work list H2D, then the mode kernels
    // on parallel branches joined back into the slot's stream
    cudaStream_t side[kModes];
    cudaEvent_t fork = nullptr, join[kModes];
    for (int m = 0; m < kModes; ++m) {
        if (cudaStreamCreateWithFlags(&side[m], cudaStreamNonBlocking) != cudaSuccess) return SLOTH_ERR_CUDA;
        cudaEventCreateWithFlags(&join[m], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    const size_t bytes = sizeof(WorkHeader) + sizeof(WorkItem) * (size_t)s->cfg.tiles_per_step;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(is.stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaMemcpyAsync(is.d_buf, is.h_buf, bytes, cudaMemcpyHostToDevice, is.stream);
        cudaEventRecord(fork, is.stream);
        const WorkItem* items = reinterpret_cast<const WorkItem*>(is.d_buf + 1);
        for (int m = 0; m < kModes; ++m) {
            cudaStreamWaitEvent(side[m], fork, 0);
            switch (m) {
                case 2 * IB_OFF: serve_kernel<IB_OFF, 0><<<blocks[m], kThreads, 0, side[m]>>>(s->d_table, is.d_buf, items, m); break;
                case 2 * IB_OFF + 1: serve_kernel<IB_OFF, 1><<<blocks[m], kThreads, 0, side[m]>>>(s->d_table, is.d_buf, items, m); break;
                case 2 * IB_SUBCRITICAL: serve_kernel<IB_SUBCRITICAL, 0><<<blocks[m], kThreads, 0, side[m]>>>(s->d_table, is.d_buf, items, m); break;
                case 2 * IB_SUBCRITICAL + 1: serve_kernel<IB_SUBCRITICAL, 1><<<blocks[m], kThreads, 0, side[m]>>>(s->d_table, is.d_buf, items, m); break;
                case 2 * IB_GENERAL: serve_kernel<IB_GENERAL, 0><<<blocks[m], kThreads, 0, side[m]>>>(s->d_table, is.d_buf, items, m); break;
                default: serve_kernel<IB_GENERAL, 1><<<blocks[m], kThreads, 0, side[m]>>>(s->d_table, is.d_buf, items, m); break;
            }
            cudaEventRecord(join[m], side[m]);
            cudaStreamWaitEvent(is.stream, join[m], 0);
        }
        e = cudaStreamEndCapture(is.stream, &graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&is.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    for (int m = 0; m < kModes; ++m) {
        cudaStreamDestroy(side[m]);
        cudaEventDestroy(join[m]);
    }
    cudaEventDestroy(fork);
    return cuda_status(e);
}

template <int IB, int FAST>
static int resident_blocks(int sms) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, serve_kernel<IB, FAST>, kThreads, 0) != cudaSuccess ||
        b < 1)
        b = 1;
    return b * sms;
}

static void grid_unref(ServerImpl* s, uint64_t key) {
    auto it = s->grids.find(key);
    if (it != s->grids.end() && it->second.refs > 0) --it->second.refs;
}

// Evicts idle grids, least recently used first, until `bytes` fit.
static bool make_room(ServerImpl* s, size_t bytes, size_t* off) {
    while (!s->arena.alloc(bytes, off)) {
        uint64_t victim = 0;
        unsigned long long oldest = ~0ull;
        bool found = false;
        for (auto& kv : s->grids) {
            if (kv.second.refs == 0 && kv.second.last_use < oldest) {
                oldest = kv.second.last_use;
                victim = kv.first;
                found = true;
            }
        }
        if (!found) return false;
        GridEntry& g = s->grids[victim];
        s->arena.release(g.off, g.bytes);
        s->grids.erase(victim);
        ++s->stats.grid_evictions;
    }
    return true;
}

static int admit_one(ServerImpl* s, Job& j) {
    if (s->free_slots.empty()) return SLOTH_ERR_BUSY;
    // grid
    GridEntry* ge = nullptr;
    auto git = s->grids.find(j.grid_key);
    if (git != s->grids.end()) {
        ge = &git->second;
    } else {
        if (!j.ne) return SLOTH_ERR_NOT_FOUND;
        const size_t gb = (size_t)j.desc.n[0] * j.desc.n[1] * j.desc.n[2] * 16u;
        size_t goff = 0;
        if (!make_room(s, gb, &goff)) return SLOTH_ERR_OUT_OF_MEMORY;
        GridEntry g;
        g.key = j.grid_key;
        g.desc = j.desc;
        g.omega = j.p.omega;
        g.off = goff;
        g.bytes = gb;
        const double nc = 3.14207787e-4 * j.p.omega * j.p.omega;
        int rc = sloth_grid_pack_trace_f32(&j.desc, j.ne, j.ne_is_f64, 1.0 / nc, j.p.ope_ratio2, s->arena.ptr(goff),
                                           s->admit);
        if (rc) {
            s->arena.release(goff, gb);
            return rc;
        }
        ++s->stats.grid_packs;
        ge = &(s->grids[j.grid_key] = g);
    }
    // job memory (the grid is pinned by a reference while we allocate)
    ++ge->refs;
    size_t parts[9];
    int bbits = 0;
    const size_t bytes = job_bytes(j.n, &j.p, &bbits, parts);
    size_t off = 0;
    if (!make_room(s, bytes, &off)) {
        --ge->refs;
        return SLOTH_ERR_OUT_OF_MEMORY;
    }
    ge->last_use = ++s->clock;
    char* base = s->arena.ptr(off);
    j.off = off;
    j.bytes = bytes;
    float* rays = reinterpret_cast<float*>(base + parts[0]);
    j.out.jones = base + parts[1];
    j.out.state = nullptr;
    j.out.phase = reinterpret_cast<double*>(base + parts[2]);
    j.out.amp = j.p.inv_brems ? base + parts[3] : nullptr;
    j.out.status = reinterpret_cast<uint8_t*>(base + parts[4]);
    j.out.steps = reinterpret_cast<int32_t*>(base + parts[5]);
    j.out.total_steps = reinterpret_cast<unsigned long long*>(base + parts[6]);
    unsigned* hist = reinterpret_cast<unsigned*>(base + parts[7]);
    const size_t an = align256((size_t)j.n * 4);
    unsigned* keys = reinterpret_cast<unsigned*>(base + parts[8]);
    unsigned* perm = reinterpret_cast<unsigned*>(base + parts[8] + an);
    unsigned* skeys = reinterpret_cast<unsigned*>(base + parts[8] + 2 * an);
    cudaError_t e = cudaMemcpyAsync(rays, j.rays_src, (size_t)j.n * 6 * 4,
                                    j.rays_on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s->admit);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, (size_t)4 << bbits, s->admit);
    if (e == cudaSuccess) e = cudaMemsetAsync(j.out.total_steps, 0, 8, s->admit);
    int rc = cuda_status(e);
    if (!rc) rc = launch_prepass<float>(&ge->desc, j.p.probing_axis, rays, j.n, bbits, keys, hist, perm, skeys,
                                        s->sms, s->admit);
    if (rc) {
        s->arena.release(off, bytes);
        --ge->refs;
        return rc;
    }
    j.slot = s->free_slots.back();
    s->free_slots.pop_back();
    TraceArgs& ta = s->h_table[j.slot];
    fill_trace_args(ta, &ge->desc, s->arena.ptr(ge->off), &j.p, rays, j.n, &j.out, perm, skeys);
    e = cudaMemcpyAsync(s->d_table + j.slot, &ta, sizeof(TraceArgs), cudaMemcpyHostToDevice, s->admit);
    if (e != cudaSuccess) return cuda_status(e);
    j.mode = 2 * trace_mode(&j.p) + (interior_sampling_ok(ta) ? 1 : 0);
    j.tiles_total = (int)((j.n + kTile - 1) / kTile);
    j.tiles_assigned = 0;
    j.state = JOB_ADMITTED;
    s->admitted.push_back(j.id);
    ++s->stats.jobs_admitted;
    return SLOTH_OK;
}

static void free_job_memory(ServerImpl* s, Job& j) {
    if (j.bytes) s->arena.release(j.off, j.bytes);
    j.bytes = 0;
    if (j.slot >= 0) s->free_slots.push_back(j.slot);
    j.slot = -1;
    grid_unref(s, j.grid_key);
}

static void retire(ServerImpl* s) {
    for (IterSlot& is : s->it) {
        if (is.iter >= 0 && cudaEventQuery(is.done) == cudaSuccess) {
            s->finished.insert(is.iter);
            float a = 0.f, b = 0.f;
            if (cudaEventElapsedTime(&a, s->t0, is.start) == cudaSuccess &&
                cudaEventElapsedTime(&b, s->t0, is.done) == cudaSuccess)
                s->intervals[is.iter] = {a, b};
            is.iter = -1;
        }
    }
    // iterations run on two streams and may finish out of order
    while (!s->finished.empty() && *s->finished.begin() == s->iter_done + 1) {
        s->iter_done = *s->finished.begin();
        s->finished.erase(s->finished.begin());
        // GPU-busy time: union of the iteration intervals, taken in iteration
        // (= start) order
        auto it = s->intervals.find(s->iter_done);
        if (it != s->intervals.end()) {
            const double a = it->second.first, b = it->second.second;
            if (s->stats.gpu_span_ms == 0.0 && s->first_start < 0.0) s->first_start = a;
            if (a >= s->busy_end) {
                s->stats.gpu_busy_ms += b - a;
            } else if (b > s->busy_end) {
                s->stats.gpu_busy_ms += b - s->busy_end;
            }
            if (b > s->busy_end) s->busy_end = b;
            s->stats.gpu_span_ms = s->busy_end - s->first_start;
            s->intervals.erase(it);
        }
    }
    cudaGetLastError();   // cudaErrorNotReady from the queries
    // jobs whose every tile ran in a finished iteration
    for (size_t i = 0; i < s->admitted.size();) {
        Job& j = s->jobs[s->admitted[i]];
        if (j.tiles_assigned == j.tiles_total && j.last_iter <= s->iter_done) {
            j.state = JOB_DONE;
            ++s->stats.jobs_done;
            s->admitted.erase(s->admitted.begin() + i);
            if (s->rr > i) --s->rr;
        } else {
            ++i;
        }
    }
    // cancelled jobs whose tiles have all run
    for (size_t i = 0; i < s->deferred.size();) {
        const DeferredFree& d = s->deferred[i];
        if (d.last_iter <= s->iter_done) {
            if (d.bytes) s->arena.release(d.off, d.bytes);
            if (d.slot >= 0) s->free_slots.push_back(d.slot);
            grid_unref(s, d.grid_key);
            s->deferred.erase(s->deferred.begin() + i);
        } else {
            ++i;
        }
    }
    // finished downloads free their memory
    for (auto& kv : s->jobs) {
        Job& j = kv.second;
        if (j.state == JOB_FETCHING && cudaEventQuery(j.fetched) == cudaSuccess) {
            j.state = JOB_FETCHED;
            free_job_memory(s, j);
        }
    }
    cudaGetLastError();
}

static int launch_iteration(ServerImpl* s) {
    IterSlot* is = nullptr;
    for (IterSlot& c : s->it)
        if (c.iter < 0) {
            is = &c;
            break;
        }
    if (!is || s->admitted.empty()) return SLOTH_OK;
    // round-robin tiles over admitted jobs
    std::vector<WorkItem> per_mode[kModes];
    const int cap = s->cfg.tiles_per_step;
    int taken = 0;
    bool any = true;
    const long long iter = s->iter_next;
    while (taken < cap && any) {
        any = false;
        for (size_t k = 0; k < s->admitted.size() && taken < cap; ++k) {
            Job& j = s->jobs[s->admitted[(s->rr + k) % s->admitted.size()]];
            int q = s->cfg.quantum;
            while (q-- > 0 && j.tiles_assigned < j.tiles_total && taken < cap) {
                per_mode[j.mode].push_back(WorkItem{j.slot, j.tiles_assigned++});
                j.last_iter = iter;
                ++taken;
                any = true;
            }
        }
    }
    if (!s->admitted.empty()) s->rr = (s->rr + 1) % s->admitted.size();
    if (taken == 0) return SLOTH_OK;
    WorkHeader* h = is->h_buf;
    memset(h, 0, sizeof(WorkHeader));
    WorkItem* items = reinterpret_cast<WorkItem*>(h + 1);
    int at = 0;
    for (int m = 0; m < kModes; ++m) {
        h->count[m] = (int)per_mode[m].size();
        h->offset[m] = at;
        for (const WorkItem& w : per_mode[m]) items[at++] = w;
    }
    cudaError_t e = cudaEventRecord(s->admit_ev, s->admit);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(is->stream, s->admit_ev, 0);
    if (e == cudaSuccess) e = cudaEventRecord(is->start, is->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(is->exec, is->stream);
    if (e == cudaSuccess) e = cudaEventRecord(is->done, is->stream);
    if (e != cudaSuccess) return cuda_status(e);
    for (int m = 0; m < kModes; ++m) {
        s->stats.kernel_launches += 1;
        note_launch();
    }
    is->iter = iter;
    ++s->iter_next;
    ++s->stats.iterations;
    s->stats.tiles += taken;
    return SLOTH_OK;
}

// Fault injection of sloth_server_create's allocations (tests): the
// allocation with this 1-based index fails once; 0 is off.
static std::atomic<int> g_fail_alloc_at{0};
constexpr int kCreateAllocs = 3 + 2 * 2;   // arena, table, pinned table, and per iteration slot two buffers

static cudaError_t create_alloc(void** p, size_t bytes, bool pinned_host, int* counter) {
    const int k = ++*counter;
    int armed = k;
    if (g_fail_alloc_at.compare_exchange_strong(armed, 0)) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return pinned_host ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes);
}

int Arena::init(size_t bytes, int* alloc_counter) {
    bytes = (bytes + 255u) & ~(size_t)255u;
    void* p = nullptr;
    cudaError_t e = create_alloc(&p, bytes, false, alloc_counter);
    if (e != cudaSuccess) {
        cudaGetLastError();
        base_ = nullptr;
        return cuda_status(e);
    }
    base_ = static_cast<char*>(p);
    size_ = bytes;
    free_.clear();
    free_[0] = bytes;
    used_ = 0;
    return SLOTH_OK;
}

}  // namespace sloth

using sloth::ServerImpl;

struct SlothServer {
    ServerImpl impl;
};

extern "C" {

int sloth_server_create(const SlothServerConfig* cfg, SlothServer** out) {
    if (!cfg || !out) return SLOTH_ERR_NULL_POINTER;
    *out = nullptr;
    if (cfg->budget_bytes < ((size_t)16 << 20) || cfg->max_jobs < 1 || cfg->max_jobs > 65536 ||
        cfg->tiles_per_step < 1 || cfg->tiles_per_step > (1 << 20) || cfg->quantum < 1)
        return SLOTH_ERR_INVALID_ARGUMENT;
    SlothServer* srv = new (std::nothrow) SlothServer();
    if (!srv) return SLOTH_ERR_OUT_OF_MEMORY;
    ServerImpl* s = &srv->impl;
    s->cfg = *cfg;
    int rc = sloth::device_sm_count(&s->sms);
    cudaError_t e = cudaGetDevice(&s->device);
    if (!rc && e != cudaSuccess) rc = sloth::cuda_status(e);
    int allocs = 0;
    if (!rc) rc = s->arena.init(cfg->budget_bytes, &allocs);
    auto fail = [&](int code) {
        sloth_server_destroy(srv);
        return code;
    };
    if (rc) return fail(rc);
    if ((e = sloth::create_alloc(reinterpret_cast<void**>(&s->d_table), sizeof(sloth::TraceArgs) * cfg->max_jobs,
                                 false, &allocs)) != cudaSuccess ||
        (e = sloth::create_alloc(reinterpret_cast<void**>(&s->h_table), sizeof(sloth::TraceArgs) * cfg->max_jobs,
                                 true, &allocs)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->admit, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->admit_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreate(&s->t0)) != cudaSuccess || (e = cudaEventRecord(s->t0, s->admit)) != cudaSuccess)
        return fail(sloth::cuda_status(e));
    for (int i = cfg->max_jobs - 1; i >= 0; --i) s->free_slots.push_back(i);
    int blocks[sloth::kModes] = {sloth::resident_blocks<sloth::IB_OFF, 0>(s->sms),
                                 sloth::resident_blocks<sloth::IB_OFF, 1>(s->sms),
                                 sloth::resident_blocks<sloth::IB_SUBCRITICAL, 0>(s->sms),
                                 sloth::resident_blocks<sloth::IB_SUBCRITICAL, 1>(s->sms),
                                 sloth::resident_blocks<sloth::IB_GENERAL, 0>(s->sms),
                                 sloth::resident_blocks<sloth::IB_GENERAL, 1>(s->sms)};
    const size_t wbytes = sizeof(sloth::WorkHeader) + sizeof(sloth::WorkItem) * (size_t)cfg->tiles_per_step;
    for (auto& is : s->it) {
        if ((e = cudaStreamCreateWithFlags(&is.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreate(&is.done)) != cudaSuccess || (e = cudaEventCreate(&is.start)) != cudaSuccess ||
            (e = sloth::create_alloc(reinterpret_cast<void**>(&is.h_buf), wbytes, true, &allocs)) != cudaSuccess ||
            (e = sloth::create_alloc(reinterpret_cast<void**>(&is.d_buf), wbytes, false, &allocs)) != cudaSuccess)
            return fail(sloth::cuda_status(e));
        memset(is.h_buf, 0, wbytes);
        if ((rc = sloth::graph_build(s, is, blocks)) != SLOTH_OK) return fail(rc);
    }
    s->stats.budget_bytes = s->arena.size();
    *out = srv;
    return SLOTH_OK;
}

int sloth_server_destroy(SlothServer* srv) {
    if (!srv) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    for (auto& is : s->it)
        if (is.stream) cudaStreamSynchronize(is.stream);
    if (s->admit) cudaStreamSynchronize(s->admit);
    if (s->copy) cudaStreamSynchronize(s->copy);
    for (auto& kv : s->jobs)
        if (kv.second.fetched) cudaEventDestroy(kv.second.fetched);
    for (auto& is : s->it) {
        if (is.exec) cudaGraphExecDestroy(is.exec);
        if (is.done) cudaEventDestroy(is.done);
        if (is.start) cudaEventDestroy(is.start);
        if (is.h_buf) cudaFreeHost(is.h_buf);
        if (is.d_buf) cudaFree(is.d_buf);
        if (is.stream) cudaStreamDestroy(is.stream);
    }
    if (s->admit_ev) cudaEventDestroy(s->admit_ev);
    if (s->t0) cudaEventDestroy(s->t0);
    if (s->admit) cudaStreamDestroy(s->admit);
    if (s->copy) cudaStreamDestroy(s->copy);
    if (s->d_table) cudaFree(s->d_table);
    if (s->h_table) cudaFreeHost(s->h_table);
    s->arena.destroy();
    cudaGetLastError();
    delete srv;
    return SLOTH_OK;
}

int sloth_server_submit(SlothServer* srv, uint64_t grid_key, const SlothGridDesc* g, const void* ne,
                        int ne_is_f64, const SlothTraceParams* p, const float* rays, int rays_on_host,
                        int64_t n, int* job_id) {
    if (!srv || !p || !job_id) return SLOTH_ERR_NULL_POINTER;
    int rc = sloth::check_trace_params(g, p, n);
    if (rc) return rc;
    if (p->integrator != SLOTH_INTEGRATOR_RKN) return SLOTH_ERR_INVALID_ARGUMENT;   // the serving kernels take RKN steps
    if (n > 0 && !rays) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    const bool resident = s->grids.count(grid_key) > 0;
    if (!resident && !ne) return SLOTH_ERR_NOT_FOUND;
    // a job that can never fit in the arena is refused now
    const size_t gb = (size_t)g->n[0] * g->n[1] * g->n[2] * 16u;
    if (sloth::job_bytes(n, p, nullptr, nullptr) + (resident ? 0 : gb) > s->arena.size()) return SLOTH_ERR_TOO_LARGE;
    if (resident && std::memcmp(&s->grids[grid_key].desc, g, sizeof(SlothGridDesc)) != 0)
        return SLOTH_ERR_INVALID_ARGUMENT;
    sloth::Job j;
    j.id = s->next_id++;
    j.grid_key = grid_key;
    j.desc = *g;
    j.ne = ne;
    j.ne_is_f64 = ne_is_f64;
    j.p = *p;
    j.rays_src = rays;
    j.rays_on_host = rays_on_host;
    j.n = n;
    if (n == 0) {
        j.state = sloth::JOB_FETCHED;
    } else {
        s->pending.push_back(j.id);
    }
    s->jobs[j.id] = j;
    ++s->stats.jobs_submitted;
    *job_id = j.id;
    return SLOTH_OK;
}

int sloth_server_step(SlothServer* srv, int* n_running, int* n_pending) {
    if (!srv) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    sloth::retire(s);
    while (!s->pending.empty()) {
        sloth::Job& j = s->jobs[s->pending.front()];
        const int rc = sloth::admit_one(s, j);
        if (rc == SLOTH_ERR_BUSY || rc == SLOTH_ERR_OUT_OF_MEMORY) break;   // wait for memory / slots
        s->pending.pop_front();
        if (rc) {
            j.state = rc;   // negative: failed
            ++s->stats.jobs_failed;
        }
    }
    const int rc = sloth::launch_iteration(s);
    if (n_running) *n_running = (int)s->admitted.size();
    if (n_pending) *n_pending = (int)s->pending.size();
    s->stats.arena_used = s->arena.used();
    s->stats.grids_resident = (long long)s->grids.size();
    return rc;
}

int sloth_server_job_state(SlothServer* srv, int job_id, int* state) {
    if (!srv || !state) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return SLOTH_ERR_NOT_FOUND;
    *state = it->second.state;
    return SLOTH_OK;
}

int sloth_server_fetch(SlothServer* srv, int job_id, const SlothTraceOutputs* dst) {
    if (!srv || !dst) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return SLOTH_ERR_NOT_FOUND;
    sloth::Job& j = it->second;
    if (j.state != sloth::JOB_DONE) return SLOTH_ERR_BUSY;
    const size_t N = (size_t)j.n, S = (size_t)j.p.n_saves;
    cudaError_t e = cudaSuccess;
    auto cp = [&](void* to, const void* from, size_t bytes) {
        if (to && from && e == cudaSuccess) e = cudaMemcpyAsync(to, from, bytes, cudaMemcpyDefault, s->copy);
    };
    cp(dst->jones, j.out.jones, S * 4 * N * 4);
    cp(dst->phase, j.out.phase, S * N * 8);
    cp(dst->amp, j.out.amp, S * N * 4);
    cp(dst->status, j.out.status, N);
    cp(dst->steps, j.out.steps, N * 4);
    cp(dst->total_steps, j.out.total_steps, 8);
    if (e == cudaSuccess && !j.fetched) e = cudaEventCreateWithFlags(&j.fetched, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(j.fetched, s->copy);
    if (e != cudaSuccess) return sloth::cuda_status(e);
    j.state = sloth::JOB_FETCHING;
    return SLOTH_OK;
}

int sloth_server_release(SlothServer* srv, int job_id) {
    if (!srv) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return SLOTH_ERR_NOT_FOUND;
    sloth::Job& j = it->second;
    if (j.state == sloth::JOB_PENDING || j.state == sloth::JOB_ADMITTED || j.state == sloth::JOB_FETCHING)
        return SLOTH_ERR_BUSY;
    if (j.state == sloth::JOB_DONE) sloth::free_job_memory(s, j);
    if (j.fetched) cudaEventDestroy(j.fetched);
    s->jobs.erase(it);
    return SLOTH_OK;
}

int sloth_server_cancel(SlothServer* srv, int job_id) {
    if (!srv) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return SLOTH_ERR_NOT_FOUND;
    sloth::Job& j = it->second;
    switch (j.state) {
        case sloth::JOB_PENDING:
            for (auto q = s->pending.begin(); q != s->pending.end(); ++q)
                if (*q == job_id) {
                    s->pending.erase(q);
                    break;
                }
            break;
        case sloth::JOB_ADMITTED: {
            // no further tiles; the memory waits for the iterations that hold
            // the tiles already handed out (last_iter), which may still run
            for (size_t i = 0; i < s->admitted.size(); ++i)
                if (s->admitted[i] == job_id) {
                    s->admitted.erase(s->admitted.begin() + i);
                    if (s->rr > i) --s->rr;
                    break;
                }
            sloth::DeferredFree d;
            d.off = j.off;
            d.bytes = j.bytes;
            d.slot = j.slot;
            d.grid_key = j.grid_key;
            d.last_iter = j.last_iter;
            s->deferred.push_back(d);
            j.bytes = 0;
            j.slot = -1;
            j.tiles_total = j.tiles_assigned;
            break;
        }
        case sloth::JOB_DONE:
            sloth::free_job_memory(s, j);
            break;
        case sloth::JOB_FETCHING:
            return SLOTH_ERR_BUSY;
        default:
            return SLOTH_OK;   // FETCHED, CANCELLED or failed: nothing to cancel
    }
    j.state = SLOTH_JOB_CANCELLED;
    ++s->stats.jobs_cancelled;
    return SLOTH_OK;
}

int sloth_server_inject_alloc_failure(int nth) {
    sloth::g_fail_alloc_at.store(nth > 0 ? nth : 0);
    return sloth::kCreateAllocs;
}

int sloth_server_stats(SlothServer* srv, SlothServerStats* st) {
    if (!srv || !st) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    std::lock_guard<std::mutex> lock(s->mu);
    s->stats.arena_used = s->arena.used();
    s->stats.grids_resident = (long long)s->grids.size();
    s->stats.cancelled_pending_free = (long long)s->deferred.size();
    *st = s->stats;
    return SLOTH_OK;
}

int sloth_server_sync(SlothServer* srv) {
    if (!srv) return SLOTH_ERR_NULL_POINTER;
    ServerImpl* s = &srv->impl;
    cudaError_t e = cudaSuccess;
    for (auto& is : s->it)
        if (e == cudaSuccess) e = cudaStreamSynchronize(is.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->admit);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy);
    return sloth::cuda_status(e);
}

}  // extern "C"
