// eb2_server.cu -- the solve server: continuous batching of independent
// solves on one GPU (include/euler_b200.h, eb2_server_*).
//
// Requests are admitted into slots while the HBM budget allows; each slot
// keeps its state, stage buffers, partials and control block on the device
// until it is retired.  All active slots advance together: one batch step is a
// CUDA graph of seven launches (boundary fill + fused stage, three times, and
// the per-slot end-of-step reduction) whose stage kernels walk the device
// work list of (slot, tile) pairs with a persistent grid.  Admission and
// retirement only rewrite the work list and descriptor arrays, so the graphs
// are reused; a graph is captured per persistent-grid size, and the size is
// picked per batch-shape class by timing the candidates (the autotuner).
// A mixed slot that fills the GPU by itself gets a stage launch of its own in
// the graph, forked beside the batched launch of the other slots.
// Every slot has its own time, CFL step and final time.
#include <algorithm>
#include <cstdarg>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <thread>
#include <vector>

#include "../../include/euler_b200.h"
#include "eb2_batch.cuh"

using namespace eb2;

namespace {

constexpr int kStepsPerGraph = 4;

struct Slot {
    bool used = false;
    bool done = false;
    long long id = -1;
    size_t bytes = 0;
    double* u = nullptr;
    double* u1 = nullptr;
    double* u2 = nullptr;
    double* partials = nullptr;
    int nx = 0, ny = 0;
    double t_final = 0.0;
    long long steps = 0;
    unsigned status = 0;
};

int fail(int code, const char* fmt, ...) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

#define CKS(expr)                                                                        \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(EB2_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_));             \
    } while (0)

// Tiles of an nx x ny slot in tile shape `shape` (32 columns per tile in
// every shape).
int slot_tiles(int nx, int ny, int precision, int shape) {
    const int tx = batch_shape_tile_x(precision, shape);
    return ((ny + STAGE_TILE_Y - 1) / STAGE_TILE_Y) * ((nx + tx - 1) / tx);
}

// Partials of a slot: one triple per tile in the shape with the most tiles (for
// the mixed form the 8-row shape, whose tiles are the 8 x 32 partial blocks).
int slot_partials(int nx, int ny, int precision) {
    int n = 296;
    for (int k = 0; k < batch_shapes(precision); k++)
        n = std::max(n, slot_tiles(nx, ny, precision, k));
    return n;
}

size_t slot_bytes(int nx, int ny, int precision) {
    size_t n = (size_t)4 * (nx + 2 * GC) * (ny + 2 * GC) * sizeof(double);
    return 3 * n + (size_t)3 * slot_partials(nx, ny, precision) * sizeof(double);
}

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct eb2_server {
    int device = 0;
    cudaStream_t stream = nullptr;
    // The server's own stream-ordered memory pool: slot buffers and work lists
    // come from it, and memory a retired slot frees stays reserved in it (up
    // to the HBM budget) for the next admission instead of being unmapped and
    // mapped again.
    cudaMemPool_t pool = nullptr;
    int precision = EB2_MIXED;
    Numerics num{};
    double gamma = 1.4;
    size_t budget = 0, used = 0;
    int nslots = 0;
    std::vector<Slot> slots;
    SlotDesc* d_desc = nullptr;
    SlotDesc* h_desc = nullptr;   // pinned
    Ctrl* d_ctrl = nullptr;
    Ctrl* h_ctrl = nullptr;       // pinned
    int2* d_work = nullptr;
    int2* h_work = nullptr;       // pinned
    int* d_nwork = nullptr;
    int* h_nwork = nullptr;       // pinned
    int work_cap = 0;
    int nwork = 0;                // work-list length in the current tile shape
    int nbatch0 = 0;              // the same in shape 0, for the batch-shape class
    int shape = 0;                // tile shape the work list is built for
    int nshapes = 1;
    int2* d_bcwork = nullptr;     // ghost-fill work list: (slot, block of the slot)
    int2* h_bcwork = nullptr;     // pinned
    int* d_counts = nullptr;      // device: ghost-fill and active-slot list lengths
    int* h_counts = nullptr;      // pinned
    int* d_active = nullptr;      // active slot indices (end-of-step reduction)
    int* h_active = nullptr;      // pinned
    int bc_cap = 0;
    bool dirty = true;
    long long next_id = 0;
    int sms = 148;
    std::map<int, cudaGraphExec_t> graphs;   // launch key (grid_key) -> graph
    std::map<int, int> tuned;                // batch-shape class -> launch key
    int bc_grid = 8;                         // blocks of the ghost-fill launches
    int active_grid = 8;                     // blocks of the end-of-step launches
    long long graph_launches = 0;
    cudaEvent_t busy0 = nullptr, busy1 = nullptr;  // around each eb2_server_step's graphs
    double busy_ms = 0.0;                    // their accumulated device time
    double tune_s = 0.0;                     // host time in autotuner trials
    double admin_s = 0.0;                    // host time in admission, rebuilds, retirement
    float last_graph_ms = 0.0f;              // device time per graph of the last step call
    // Slots that fill the GPU by themselves (a mixed slot with at least as many
    // tiles as the GPU holds CTAs of the default shape) get a stage launch of
    // their own in the graphs, beside the batched launch of the other slots:
    // their stage arguments then sit in the kernel's parameter block instead
    // of being copied to shared memory per CTA.  They stay in the ghost-fill
    // and end-of-step lists.
    std::vector<int> own;                    // their slot indices
    std::vector<long long> own_ids;          // and request ids (a slot index is reused)
    static constexpr int kSide = 4;          // streams their launches fork onto
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kSide] = {};
};

namespace {
// Adds the wall time of a scope to a server counter.
struct HostTimer {
    double& acc;
    double t0;
    explicit HostTimer(double& a) : acc(a), t0(now_s()) {}
    ~HostTimer() { acc += now_s() - t0; }
};
}  // namespace

namespace {

void destroy_graphs(eb2_server* s) {
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
}

cudaError_t stage_batch(eb2_server* s, const BatchLaunch& b, int stage) {
    return s->precision == EB2_MIXED ? launch_stage_batch_mixed(b, s->num, stage, s->stream)
                                     : launch_stage_batch_fp64(b, s->num, stage, s->stream);
}

// A stage-kernel launch shape: tile shape `shape`, `grid` CTAs looping over the
// work list (each = 0) or one per work item (each = 1, grid >= the work-list
// length).
int grid_key(int shape, int grid, int each) { return (shape << 24) | (2 * grid + each); }

int get_graph(eb2_server* s, int key, cudaGraphExec_t* out) {
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = it->second;
        return EB2_OK;
    }
    BatchLaunch b{s->d_desc, s->nslots, s->d_work, s->d_nwork, 0,
                  s->d_bcwork, s->d_counts, s->bc_grid,
                  s->d_active, s->d_counts + 1, s->active_grid};
    b.shape = key >> 24;
    CKS(stage_batch(s, b, 0));  // kernel attributes, outside the capture
    if (!s->own.empty()) {
        StageArgs cfg = slot_args(s->h_desc[s->own[0]], 0);
        cfg.uout = nullptr;  // configuration only
        CKS(launch_stage_slot_mixed(cfg, s->num, b.shape, s->stream));
    }
    b.grid = (key & 0xffffff) / 2;
    b.each = key % 2;
    cudaGraph_t g = nullptr;
    CKS(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    const int nside = std::min<int>((int)s->own.size(), eb2_server::kSide);
    for (int k = 0; k < kStepsPerGraph && !e; k++) {
        for (int st = 0; st < 3 && !e; st++) {
            e = launch_bc_batch(b, st, s->stream);
            // the slots with launches of their own run beside the batched launch
            if (!e && nside) e = cudaEventRecord(s->fork, s->stream);
            for (int j = 0; j < nside && !e; j++) e = cudaStreamWaitEvent(s->side[j], s->fork, 0);
            for (size_t q = 0; q < s->own.size() && !e; q++)
                e = launch_stage_slot_mixed(slot_args(s->h_desc[s->own[q]], st), s->num,
                                            b.shape, s->side[q % eb2_server::kSide]);
            if (!e) e = stage_batch(s, b, st);
            for (int j = 0; j < nside && !e; j++) {
                e = cudaEventRecord(s->join[j], s->side[j]);
                if (!e) e = cudaStreamWaitEvent(s->stream, s->join[j], 0);
            }
        }
        if (!e) e = launch_finalize_batch(b, s->stream);
    }
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    if (e || e2) {
        if (g) cudaGraphDestroy(g);
        return fail(EB2_ECUDA, "batch graph capture: %s", cudaGetErrorString(e ? e : e2));
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e) return fail(EB2_ECUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
    s->graphs[key] = ex;
    *out = ex;
    return EB2_OK;
}

// Rewrite the work list and descriptors after admissions and retirements.
int rebuild(eb2_server* s) {
    HostTimer timer(s->admin_s);
    std::vector<int> own;
    std::vector<long long> own_ids;
    const int fills = s->sms * stage_batch_max_blocks_per_sm(1, 0);
    int n = 0, nb0 = 0;
    for (int q = 0; q < s->nslots; q++)
        if (s->slots[q].used && !s->slots[q].done) {
            if (s->precision == EB2_MIXED && s->h_desc[q].ntiles[0] >= fills) {
                own.push_back(q);
                own_ids.push_back(s->slots[q].id);
            } else {
                n += s->h_desc[q].ntiles[s->shape];
                nb0 += s->h_desc[q].ntiles[0];
            }
        }
    s->nbatch0 = nb0;
    if (own_ids != s->own_ids) {
        // the graphs hold the own launches' arguments, buffer addresses included:
        // a new request in a reused slot index has buffers of its own
        s->own = own;
        s->own_ids = own_ids;
        destroy_graphs(s);
    }
    if (n > s->work_cap) {
        int cap = std::max(n, 2 * s->work_cap);
        if (s->d_work) CKS(cudaFreeAsync(s->d_work, s->stream));
        if (s->h_work) {
            CKS(cudaStreamSynchronize(s->stream));
            cudaFreeHost(s->h_work);
        }
        CKS(cudaMallocFromPoolAsync(&s->d_work, (size_t)cap * sizeof(int2), s->pool, s->stream));
        CKS(cudaMallocHost(&s->h_work, (size_t)cap * sizeof(int2)));
        s->work_cap = cap;
        destroy_graphs(s);  // graphs hold the old work-list address
    }
    // ghost-fill blocks: each active slot takes enough 256-thread blocks for its
    // 32 (nx + ny) ghost values (at most 256; the blocks loop beyond that)
    int nbc = 0, nact = 0;
    for (int q = 0; q < s->nslots; q++)
        if (s->slots[q].used && !s->slots[q].done) {
            const Grid& g = s->h_desc[q].grid;
            s->h_desc[q].bc_blocks =
                (int)std::min<long long>((32LL * (g.nx + g.ny) + 255) / 256, 256);
            nbc += s->h_desc[q].bc_blocks;
            nact++;
        }
    if (nbc > s->bc_cap) {
        int cap = std::max(nbc, 2 * s->bc_cap);
        if (s->d_bcwork) CKS(cudaFreeAsync(s->d_bcwork, s->stream));
        if (s->h_bcwork) {
            CKS(cudaStreamSynchronize(s->stream));
            cudaFreeHost(s->h_bcwork);
        }
        CKS(cudaMallocFromPoolAsync(&s->d_bcwork, (size_t)cap * sizeof(int2), s->pool,
                                    s->stream));
        CKS(cudaMallocHost(&s->h_bcwork, (size_t)cap * sizeof(int2)));
        s->bc_cap = cap;
        destroy_graphs(s);  // graphs hold the old list address
    }
    // launch grids: powers of two covering the lists, so that graphs are only
    // captured again when a list outgrows its grid
    auto pow2 = [](int n) {
        int g = 8;
        while (g < n) g *= 2;
        return g;
    };
    const int bc_grid = pow2(nbc), active_grid = pow2(nact);
    if (bc_grid != s->bc_grid || active_grid != s->active_grid) {
        s->bc_grid = bc_grid;
        s->active_grid = active_grid;
        destroy_graphs(s);  // graphs hold the launch grids
    }
    CKS(cudaStreamSynchronize(s->stream));  // the pinned staging arrays are reused
    int w = 0;
    for (int q = 0; q < s->nslots; q++) {
        if (!s->slots[q].used || s->slots[q].done) continue;
        if (std::find(s->own.begin(), s->own.end(), q) != s->own.end()) continue;
        for (int t = 0; t < s->h_desc[q].ntiles[s->shape]; t++) s->h_work[w++] = make_int2(q, t);
    }
    *s->h_nwork = w;
    s->nwork = w;
    int nb = 0, na = 0;
    for (int q = 0; q < s->nslots; q++) {
        if (!s->slots[q].used || s->slots[q].done) continue;
        for (int k = 0; k < s->h_desc[q].bc_blocks; k++) s->h_bcwork[nb++] = make_int2(q, k);
        s->h_active[na++] = q;
    }
    s->h_counts[0] = nb;
    s->h_counts[1] = na;
    if (w) CKS(cudaMemcpyAsync(s->d_work, s->h_work, (size_t)w * sizeof(int2),
                               cudaMemcpyHostToDevice, s->stream));
    CKS(cudaMemcpyAsync(s->d_nwork, s->h_nwork, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    if (nb) CKS(cudaMemcpyAsync(s->d_bcwork, s->h_bcwork, (size_t)nb * sizeof(int2),
                                cudaMemcpyHostToDevice, s->stream));
    if (na) CKS(cudaMemcpyAsync(s->d_active, s->h_active, (size_t)na * sizeof(int),
                                cudaMemcpyHostToDevice, s->stream));
    CKS(cudaMemcpyAsync(s->d_counts, s->h_counts, 2 * sizeof(int), cudaMemcpyHostToDevice,
                        s->stream));
    CKS(cudaMemcpyAsync(s->d_desc, s->h_desc, (size_t)s->nslots * sizeof(SlotDesc),
                        cudaMemcpyHostToDevice, s->stream));
    s->dirty = false;
    return EB2_OK;
}

int shape_class(int nwork) {
    int c = 0;
    while ((1 << c) < nwork) c++;
    return c;
}

// The batch-shape class the autotuner keys on: log2 of the batched work-list
// length in shape 0 (the slots with launches of their own are not in it).
int batch_class(const eb2_server* s) { return shape_class(s->nbatch0); }

// Switch the work list to tile shape `shape`.
int use_shape(eb2_server* s, int shape) {
    if (shape == s->shape && !s->dirty) return EB2_OK;
    s->shape = shape;
    return rebuild(s);
}

// One graph launch (kStepsPerGraph batch steps) with the tuned launch shape.
// The autotuner times, per batch-shape class (log2 of the batched work-list
// length in tile shape 0), every tile shape of the server's form and, per tile shape,
// persistent grids of 1..CTAS CTAs per SM smaller than the work list and one
// CTA per work item; the fastest is kept for the class.
int launch_steps(eb2_server* s) {
    const int prec = s->precision == EB2_MIXED ? 1 : 0;
    const int cls = batch_class(s);
    auto it = s->tuned.find(cls);
    if (it == s->tuned.end()) {
        HostTimer timer(s->tune_s);
        // the slots advance during the trials, which is ordinary progress
        int best = 0;
        float best_ms = 1e30f;
        cudaEvent_t e0, e1;
        CKS(cudaEventCreate(&e0));
        CKS(cudaEventCreate(&e1));
        for (int sh = 0; sh < s->nshapes; sh++) {
            if (int r = use_shape(s, sh)) return r;
            // one CTA per work item over 2^k CTAs covers every work-list length
            // of this class in this shape (an 8-row tile shape has up to twice
            // the tiles of shape 0, a 32-row one at most as many)
            const int each_grid = 1 << (shape_class(s->nbatch0) +
                                        (batch_shape_tile_x(prec, sh) <
                                         batch_shape_tile_x(prec, 0) ? 1 : 0));
            // persistent grids are tried in the default shape only: the trials
            // cost host time (a capture each) and progress at a worse rate
            std::vector<int> keys;
            if (sh == 0)
                for (int mult = 1; mult <= stage_batch_max_blocks_per_sm(prec, sh); mult++)
                    if (mult * s->sms < s->nwork) keys.push_back(grid_key(sh, mult * s->sms, 0));
            keys.push_back(grid_key(sh, each_grid, 1));
            for (int key : keys) {
                cudaGraphExec_t ex;
                if (int r = get_graph(s, key, &ex)) return r;
                // one untimed launch first: the first launch of a new graph also
                // uploads it, which would bias the comparison by more than the
                // candidates differ
                CKS(cudaGraphLaunch(ex, s->stream));
                s->graph_launches++;
                CKS(cudaEventRecord(e0, s->stream));
                CKS(cudaGraphLaunch(ex, s->stream));
                CKS(cudaEventRecord(e1, s->stream));
                CKS(cudaEventSynchronize(e1));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                s->graph_launches++;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = key;
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        s->tuned[cls] = best;
        return use_shape(s, best >> 24);
    }
    if (int r = use_shape(s, it->second >> 24)) return r;
    cudaGraphExec_t ex;
    if (int r = get_graph(s, it->second, &ex)) return r;
    CKS(cudaGraphLaunch(ex, s->stream));
    s->graph_launches++;
    return EB2_OK;
}

// Read every slot's control block; mark the finished ones.
int harvest(eb2_server* s, int* nfinished) {
    CKS(cudaMemcpyAsync(s->h_ctrl, s->d_ctrl, (size_t)s->nslots * sizeof(Ctrl),
                        cudaMemcpyDeviceToHost, s->stream));
    CKS(cudaStreamSynchronize(s->stream));
    int n = 0;
    for (int q = 0; q < s->nslots; q++) {
        Slot& sl = s->slots[q];
        if (!sl.used || sl.done) continue;
        const Ctrl& c = s->h_ctrl[q];
        if (!c.active) {
            sl.done = true;
            sl.t_final = c.t;
            sl.steps = c.step;
            sl.status = c.status;
            s->dirty = true;
            n++;
        }
    }
    if (nfinished) *nfinished = n;
    return EB2_OK;
}

int find_slot(eb2_server* s, long long id) {
    for (int q = 0; q < s->nslots; q++)
        if (s->slots[q].used && s->slots[q].id == id) return q;
    return -1;
}

}  // namespace

extern "C" {

int eb2_server_create(eb2_server** out, int device, int max_slots,
                      unsigned long long hbm_budget_bytes, int precision, int recon,
                      int characteristic, int weno_z, int scheme, double gamma) {
    if (!out) return fail(EB2_EARG, "null output");
    *out = nullptr;
    if (max_slots < 1 || max_slots > 65535) return fail(EB2_EARG, "max_slots out of range");
    if (precision != EB2_FP64 && precision != EB2_MIXED) return fail(EB2_EARG, "precision");
    if (recon != 5) return fail(EB2_EUNSUPPORTED, "the server runs WENO5 reconstructions");
    if (precision == EB2_MIXED && !characteristic)
        return fail(EB2_EUNSUPPORTED, "the mixed form reconstructs in characteristic variables");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(EB2_ECUDA, "no CUDA device available; there is no CPU path");
    if (device < 0 || device >= ndev) return fail(EB2_EARG, "device out of range");
    CKS(cudaSetDevice(device));
    eb2_server* s = new (std::nothrow) eb2_server();
    if (!s) return fail(EB2_ENOMEM, "host allocation failed");
    s->device = device;
    s->precision = precision;
    s->num.recon = recon;
    s->num.characteristic = characteristic ? 1 : 0;
    s->num.weno_z = weno_z ? 1 : 0;
    s->num.flux = scheme == 1    ? FLUX_HLL
                  : scheme == 2  ? FLUX_HLLC
                  : scheme == 3  ? FLUX_ROE
                  : scheme == 11 ? FLUX_HLLHC
                  : scheme == 22 ? FLUX_HLLCHC
                  : scheme == 33 ? FLUX_ROEHC
                                 : FLUX_LLF;
    s->gamma = gamma;
    s->nshapes = batch_shapes(precision == EB2_MIXED ? 1 : 0);
    s->budget = hbm_budget_bytes;
    s->nslots = max_slots;
    s->slots.resize(max_slots);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
    auto bail = [&](int code) {
        eb2_server_destroy(s);
        return code;
    };
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    unsigned long long keep = hbm_budget_bytes;
    if (cudaMemPoolCreate(&s->pool, &props) ||
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep))
        return bail(fail(EB2_ECUDA, "server memory pool"));
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) ||
        cudaMalloc(&s->d_desc, (size_t)max_slots * sizeof(SlotDesc)) ||
        cudaMallocHost(&s->h_desc, (size_t)max_slots * sizeof(SlotDesc)) ||
        cudaMalloc(&s->d_ctrl, (size_t)max_slots * sizeof(Ctrl)) ||
        cudaMallocHost(&s->h_ctrl, (size_t)max_slots * sizeof(Ctrl)) ||
        cudaMalloc(&s->d_nwork, sizeof(int)) || cudaMallocHost(&s->h_nwork, sizeof(int)) ||
        cudaMalloc(&s->d_counts, 2 * sizeof(int)) ||
        cudaMallocHost(&s->h_counts, 2 * sizeof(int)) ||
        cudaMalloc(&s->d_active, (size_t)max_slots * sizeof(int)) ||
        cudaMallocHost(&s->h_active, (size_t)max_slots * sizeof(int)))
        return bail(fail(EB2_ENOMEM, "server allocation failed"));
    if (cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming))
        return bail(fail(EB2_ECUDA, "server events"));
    for (int j = 0; j < eb2_server::kSide; j++)
        if (cudaStreamCreateWithFlags(&s->side[j], cudaStreamNonBlocking) ||
            cudaEventCreateWithFlags(&s->join[j], cudaEventDisableTiming))
            return bail(fail(EB2_ECUDA, "server streams"));
    memset(s->h_desc, 0, (size_t)max_slots * sizeof(SlotDesc));
    if (cudaMemsetAsync(s->d_ctrl, 0, (size_t)max_slots * sizeof(Ctrl), s->stream) ||
        cudaMemcpyAsync(s->d_desc, s->h_desc, (size_t)max_slots * sizeof(SlotDesc),
                        cudaMemcpyHostToDevice, s->stream) ||
        cudaStreamSynchronize(s->stream))
        return bail(fail(EB2_ECUDA, "server initialisation failed"));
    *out = s;
    return EB2_OK;
}

int eb2_server_destroy(eb2_server* s) {
    if (!s) return EB2_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    destroy_graphs(s);
    if (s->busy0) cudaEventDestroy(s->busy0);
    if (s->busy1) cudaEventDestroy(s->busy1);
    for (int j = 0; j < eb2_server::kSide; j++) {
        if (s->side[j]) cudaStreamSynchronize(s->side[j]);
        if (s->side[j]) cudaStreamDestroy(s->side[j]);
        if (s->join[j]) cudaEventDestroy(s->join[j]);
    }
    if (s->fork) cudaEventDestroy(s->fork);
    for (auto& sl : s->slots)
        if (sl.used) {
            cudaFree(sl.u);
            cudaFree(sl.u1);
            cudaFree(sl.u2);
            cudaFree(sl.partials);
        }
    cudaFree(s->d_desc);
    cudaFreeHost(s->h_desc);
    cudaFree(s->d_ctrl);
    cudaFreeHost(s->h_ctrl);
    cudaFree(s->d_work);
    cudaFreeHost(s->h_work);
    cudaFree(s->d_nwork);
    cudaFreeHost(s->h_nwork);
    cudaFree(s->d_bcwork);
    cudaFreeHost(s->h_bcwork);
    cudaFree(s->d_counts);
    cudaFreeHost(s->h_counts);
    cudaFree(s->d_active);
    cudaFreeHost(s->h_active);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return EB2_OK;
}

int eb2_server_submit(eb2_server* s, const eb2_request* r, long long* id) {
    if (!s || !r) return fail(EB2_EARG, "null argument");
    HostTimer timer(s->admin_s);
    if (r->nx < 1 || r->ny < 1) return fail(EB2_EARG, "empty grid");
    CKS(cudaSetDevice(s->device));
    InitDesc d;
    double L[2], T;
    int bc[4];
    if (int rc = case_setup(r->test_case, r->has_q ? r->q : nullptr, d, L, T, bc)) return rc;
    if (r->lx > 0.0) L[0] = d.lx = r->lx;
    if (r->ly > 0.0) L[1] = d.ly = r->ly;
    if (r->tmax > 0.0) T = r->tmax;
    for (int q = 0; q < 4; q++) {
        int n = q < 2 ? r->nx : r->ny;
        if ((bc[q] == BC_PERIODIC || (bc[q] == BC_REFLECT && (q == 0 || q == 3))) && n < GC)
            return fail(EB2_EUNSUPPORTED, "mirrored or periodic side needs 4 interior cells");
    }
    const size_t bytes = slot_bytes(r->nx, r->ny, s->precision == EB2_MIXED ? 1 : 0);
    if (s->used + bytes > s->budget) return fail(EB2_EBUSY, "HBM budget exhausted");
    int q = -1;
    for (int k = 0; k < s->nslots; k++)
        if (!s->slots[k].used) {
            q = k;
            break;
        }
    if (q < 0) return fail(EB2_EBUSY, "no free slot");
    Slot& sl = s->slots[q];
    const int rows = r->nx + 2 * GC, cols = r->ny + 2 * GC;
    const size_t n = (size_t)4 * rows * cols * sizeof(double);
    const int prec = s->precision == EB2_MIXED ? 1 : 0;
    const int npart = slot_partials(r->nx, r->ny, prec);
    // Any failure from here on releases what this call allocated and leaves
    // the slot unused, so that a failed admission leaks nothing.
    auto undo = [&](int code) {
        double** bufs[4] = {&sl.u, &sl.u1, &sl.u2, &sl.partials};
        for (double** b : bufs)
            if (*b) {
                cudaFreeAsync(*b, s->stream);
                *b = nullptr;
            }
        cudaStreamSynchronize(s->stream);
        memset(&s->h_desc[q], 0, sizeof(SlotDesc));
        sl = Slot();
        return code;
    };
#define CKU(expr)                                                                        \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return undo(fail(EB2_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_)));       \
    } while (0)
    CKU(cudaMallocFromPoolAsync(&sl.u, n, s->pool, s->stream));
    CKU(cudaMallocFromPoolAsync(&sl.u1, n, s->pool, s->stream));
    CKU(cudaMallocFromPoolAsync(&sl.u2, n, s->pool, s->stream));
    CKU(cudaMallocFromPoolAsync(&sl.partials, (size_t)3 * npart * sizeof(double), s->pool,
                                s->stream));
    CKU(cudaMemsetAsync(sl.u, 0, n, s->stream));
    CKU(cudaMemsetAsync(sl.u1, 0, n, s->stream));
    CKU(cudaMemsetAsync(sl.u2, 0, n, s->stream));
    SlotDesc& sd = s->h_desc[q];
    memset(&sd, 0, sizeof sd);
    sd.u = sl.u;
    sd.u1 = sl.u1;
    sd.u2 = sl.u2;
    sd.partials = sl.partials;
    sd.ctrl = s->d_ctrl + q;
    sd.grid.nx = r->nx;
    sd.grid.ny = r->ny;
    sd.grid.rows = rows;
    sd.grid.cols = cols;
    sd.grid.dx = L[0] / r->nx;
    sd.grid.dy = L[1] / r->ny;
    sd.grid.inv_dx = 1.0 / sd.grid.dx;
    sd.grid.inv_dy = 1.0 / sd.grid.dy;
    sd.gas = Gas{s->gamma, s->gamma - 1.0, s->gamma / (s->gamma - 1.0)};
    sd.num = s->num;
    const double mach3[4] = {1.4, 1.4 * 3.0, 0.0, 1.0 / 0.4 + 0.5 * 1.4 * 3.0 * 3.0};
    for (int k = 0; k < 4; k++) {
        sd.bnd.kind[k] = bc[k];
        sd.bnd.inflow[k] = mach3[k];
        for (int m = 0; m < 4; m++) sd.bnd.fixed[m][k] = mach3[k];
    }
    sd.tiles_x = (r->ny + STAGE_TILE_Y - 1) / STAGE_TILE_Y;
    for (int k = 0; k < s->nshapes; k++) sd.ntiles[k] = slot_tiles(r->nx, r->ny, prec, k);
    sd.ncells = r->nx * r->ny;
    sd.npartials = prec ? sd.tiles_x * ((r->nx + MIXED_PARTIAL_ROWS - 1) / MIXED_PARTIAL_ROWS)
                        : sd.ntiles[0];
    CKU(launch_init(sl.u, sd.grid, sd.gas, d, s->stream));
    // control block and first CFL step, as eb2_run starts a solve
    const double cfl = r->cfl > 0.0 ? r->cfl : 0.5;
    const double dmin = sd.grid.dx > sd.grid.dy ? sd.grid.dy : sd.grid.dx;
    CKU(cudaMemsetAsync(s->d_ctrl + q, 0, sizeof(Ctrl), s->stream));
    set_loop_ctrl(s->d_ctrl + q, 0.0, T, T, cfl, dmin, LLONG_MAX, s->stream);
    CKU(cudaGetLastError());
    int nb = 0;
    CKU(launch_wave_partials(sl.u, sd.grid, sd.gas, sl.partials, &nb, s->stream));
    CKU(launch_finalize(s->d_ctrl + q, sl.partials, nb, sd.ncells, 1, s->stream));
#undef CKU
    sl.used = true;
    sl.done = false;
    sl.id = s->next_id++;
    sl.bytes = bytes;
    sl.nx = r->nx;
    sl.ny = r->ny;
    s->used += bytes;
    s->dirty = true;
    if (id) *id = sl.id;
    return EB2_OK;
}

int eb2_server_step(eb2_server* s, int ngraphs, int* nfinished) {
    if (!s) return fail(EB2_EARG, "null server");
    CKS(cudaSetDevice(s->device));
    if (s->dirty)
        if (int r = rebuild(s)) return r;
    if (nfinished) *nfinished = 0;
    if (s->nwork == 0 && s->own.empty()) return EB2_OK;  // no active slot
    if (!s->busy0) {
        CKS(cudaEventCreate(&s->busy0));
        CKS(cudaEventCreate(&s->busy1));
    }
    CKS(cudaEventRecord(s->busy0, s->stream));
    const long long launched = s->graph_launches;
    for (int k = 0; k < ngraphs; k++)
        if (int r = launch_steps(s)) return r;
    CKS(cudaEventRecord(s->busy1, s->stream));
    int r = harvest(s, nfinished);  // synchronizes the stream
    float ms = 0.0f;
    if (!r && cudaEventElapsedTime(&ms, s->busy0, s->busy1) == cudaSuccess) {
        s->busy_ms += ms;
        // (not when autotuner trials ran in this call)
        if (s->graph_launches - launched == ngraphs && ngraphs > 0)
            s->last_graph_ms = ms / (float)ngraphs;
    }
    return r;
}

// Device time of the batch steps so far (the graphs of every eb2_server_step),
// and the host time spent in autotuner trials and in admission, rebuilds and
// retirement.
int eb2_server_timing(eb2_server* s, double* busy_ms, double* tune_s, double* admin_s) {
    if (!s) return fail(EB2_EARG, "null server");
    if (busy_ms) *busy_ms = s->busy_ms;
    if (tune_s) *tune_s = s->tune_s;
    if (admin_s) *admin_s = s->admin_s;
    return EB2_OK;
}

int eb2_server_poll(eb2_server* s, long long* ids, double* t_final, long long* steps,
                    unsigned* status, int max, int* n) {
    if (!s || !n) return fail(EB2_EARG, "null argument");
    int k = 0;
    for (int q = 0; q < s->nslots && k < max; q++) {
        const Slot& sl = s->slots[q];
        if (!sl.used || !sl.done) continue;
        if (ids) ids[k] = sl.id;
        if (t_final) t_final[k] = sl.t_final;
        if (steps) steps[k] = sl.steps;
        if (status) status[k] = sl.status;
        k++;
    }
    *n = k;
    return EB2_OK;
}

int eb2_server_fetch(eb2_server* s, long long id, double* U) {
    if (!s) return fail(EB2_EARG, "null server");
    HostTimer timer(s->admin_s);
    CKS(cudaSetDevice(s->device));
    int q = find_slot(s, id);
    if (q < 0) return fail(EB2_EARG, "unknown request id %lld", id);
    Slot& sl = s->slots[q];
    if (!sl.done) return fail(EB2_EBUSY, "request %lld has not finished", id);
    if (U) {
        const size_t n = (size_t)4 * (sl.nx + 2 * GC) * (sl.ny + 2 * GC) * sizeof(double);
        CKS(cudaMemcpyAsync(U, sl.u, n, cudaMemcpyDeviceToHost, s->stream));
    }
    CKS(cudaFreeAsync(sl.u, s->stream));
    CKS(cudaFreeAsync(sl.u1, s->stream));
    CKS(cudaFreeAsync(sl.u2, s->stream));
    CKS(cudaFreeAsync(sl.partials, s->stream));
    CKS(cudaStreamSynchronize(s->stream));
    memset(&s->h_desc[q], 0, sizeof(SlotDesc));
    s->used -= sl.bytes;
    sl = Slot();
    s->dirty = true;
    return EB2_OK;
}

int eb2_server_stats(eb2_server* s, unsigned long long* hbm_used, int* active,
                     long long* graph_launches) {
    if (!s) return fail(EB2_EARG, "null server");
    int a = 0;
    for (const Slot& sl : s->slots) a += sl.used && !sl.done;
    if (hbm_used) *hbm_used = s->used;
    if (active) *active = a;
    if (graph_launches) *graph_launches = s->graph_launches;
    return EB2_OK;
}

// Replay a request trace in real time: requests arrive at arrival_s[i]
// seconds after the call starts, wait in FIFO order until a slot and the HBM
// budget admit them, run in the batch, and are retired as they finish.
int eb2_server_run_trace(eb2_server* s, const eb2_request* reqs, const double* arrival_s, int n,
                         double* admit_s, double* finish_s, long long* steps, unsigned* status,
                         double** results, double* makespan_s) {
    if (!s || (!reqs && n) || (!arrival_s && n)) return fail(EB2_EARG, "null argument");
    CKS(cudaSetDevice(s->device));
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return arrival_s[a] < arrival_s[b]; });
    std::map<long long, int> owner;  // request id -> trace index
    std::vector<int> queue;
    size_t next = 0, qhead = 0;
    int completed = 0;
    const double t0 = now_s();
    while (completed < n) {
        double t = now_s() - t0;
        while (next < order.size() && arrival_s[order[next]] <= t) queue.push_back(order[next++]);
        while (qhead < queue.size()) {
            long long id;
            int i = queue[qhead];
            int rc = eb2_server_submit(s, &reqs[i], &id);
            if (rc == EB2_EBUSY) break;
            if (rc) return rc;
            owner[id] = i;
            if (admit_s) admit_s[i] = now_s() - t0;
            qhead++;
        }
        int active = 0;
        for (const Slot& sl : s->slots) active += sl.used && !sl.done;
        if (!active) {
            if (qhead < queue.size()) return fail(EB2_EBUSY, "a request never fits the budget");
            if (next < order.size()) {
                double wait = arrival_s[order[next]] - (now_s() - t0);
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
            }
            continue;
        }
        int nf = 0;
        // enough graphs per call that the GPU works ~2 ms between the host's
        // harvests (a small batch's graph takes a fraction of that, and the
        // host's admission and retirement work would otherwise leave it idle),
        // from the device time per graph of the last call
        int ngraphs = 1;
        if (s->last_graph_ms > 0.0f)
            ngraphs = std::max(1, std::min(16, (int)(2.0f / s->last_graph_ms)));
        if (int rc = eb2_server_step(s, ngraphs, &nf)) return rc;
        if (!nf) continue;
        const double tf = now_s() - t0;
        for (int q = 0; q < s->nslots; q++) {
            Slot& sl = s->slots[q];
            if (!sl.used || !sl.done) continue;
            int i = owner[sl.id];
            if (finish_s) finish_s[i] = tf;
            if (steps) steps[i] = sl.steps;
            if (status) status[i] = sl.status;
            if (int rc = eb2_server_fetch(s, sl.id, results ? results[i] : nullptr)) return rc;
            completed++;
        }
    }
    if (makespan_s) *makespan_s = now_s() - t0;
    return EB2_OK;
}

}  // extern "C"
