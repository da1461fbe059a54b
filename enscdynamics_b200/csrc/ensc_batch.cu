// Batched stepping of many independent solver instances (ensc_batch_* in
// include/ensc_gpu.h).
//
// Instances are sub-allocated from a CUDA memory pool owned by the batch (the
// arena, bounded by a byte budget); each keeps the single-instance layout of
// ensc_instance.h in its block.  A device table of instance descriptors and
// two tile lists (32-element and 32-node tiles, each inside one instance)
// drive one persistent launch per phase for all instances, each with its own
// clock, dt and material.  The cycle is captured once as a CUDA graph; adding
// or removing instances rewrites the tables in place, so the graph stays
// valid.  Instances advance until their own cycle budget or end time, then
// idle (their tiles return at once) until the host retires them.
#include "ensc_gpu.h"
#include "ensc_device.cuh"
#include "ensc_instance.h"
#include "ensc_kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using ensc::Ctl;

namespace {

struct Slot {
    bool used = false;
    void* block = nullptr;
    size_t bytes = 0;
    int64_t nn = 0, ne = 0, nn_pad = 0, ne_pad = 0;
    bool plastic = false;
    ensc::ElemArrays E{};
    ensc::NodeArrays N{};
    ensc::PatchArrays PA{};
    ensc::Material M{};
    bool kinetic0_done = false;
    double* amp = nullptr;  // gravity amplitude table (from the pool)
    // added, with its device work on the admission stream, and not yet
    // joined by the batch stream
    bool pending = false;
};

// Launch choices of the batched cycle: grid multipliers (over one wave of
// resident blocks) of the element and node passes, cycles per graph launch,
// and threads per block of the node pass.
struct Tune {
    int mult_e = 1, mult_n = 1, chunk = 32, node_threads = ensc::kNodeThreads;
    int ept = 1;  // elements per thread of the element pass
};

}  // namespace

struct ensc_batch {
    int device = 0;
    int precision = ENSC_MIXED;
    int assembly = ENSC_ASSEMBLY_AUTO;  // for ensc_batch_add
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t cap_stream = nullptr;
    // admission stream: the device work of adding an instance (upload, init
    // pass, its boundary conditions and arming until the batch stream joins)
    // runs here, so that it overlaps the cycles the batch stream runs;
    // side_done marks the end of the work enqueued on it so far
    cudaStream_t side = nullptr;
    cudaEvent_t side_done = nullptr;
    bool side_work = false;   // side work enqueued since the batch stream last joined
    cudaMemPool_t pool = nullptr;
    int64_t budget = 0, used = 0;
    int slots = 0;
    int64_t max_etiles = 0, max_ntiles = 0;
    int etile = 32, ntile = 32;   // elements / nodes per tile
    // device tables (one allocation)
    void* tables = nullptr;
    ensc::InstanceDesc* d_desc = nullptr;
    int32_t *d_etile_inst = nullptr, *d_etile_base = nullptr, *d_ntile_inst = nullptr, *d_ntile_base = nullptr;
    int32_t* d_counts = nullptr;   // [0..2] tile and slot counts, [3] edge-prepass counter
    double *d_etile_part = nullptr, *d_ntile_part = nullptr;
    Ctl* d_ctl = nullptr;
    double* d_scratch = nullptr;  // partials for init / kinetic passes of one instance
    ensc::NodeParam* d_nparam = nullptr;
    ensc::StageHdr* d_sparam = nullptr;
    ensc::NodeView* d_nview = nullptr;
    ensc::ETileSrc* d_etile_src = nullptr;
    int scratch_blocks = 4096;
    Ctl* h_ctl = nullptr;         // pinned mirror of d_ctl
    std::vector<Slot> inst;
    ensc::BatchTables T{};
    bool dirty = true;
    ensc::InstanceDesc h_desc_off{};  // host copy of a removed slot's table entry
    int64_t n_etiles = 0, n_ntiles = 0;
    int sms = 148, occ_e = 1, occ_pre = 4;
    Tune tune;
    int fixed_chunk = 0;  // cycles per graph launch given by the caller (0: tuned)
    bool tuned = false;
    // tuning in progress: next candidate, best time per cycle and its choice;
    // element tiles of the batch the last tuning measured
    int tune_next = 0;
    float tune_best = 1e30f;
    Tune tune_pick;
    int64_t tune_etiles = 0;
    int tunings = 0;  // completed tunings
    cudaGraphExec_t graph = nullptr;
    int graph_chunk = 0, graph_ge = 0, graph_gn = 0, graph_nt = 0, graph_ept = 0;
    int occ_e2 = 1;  // resident element-pass blocks per SM at 2 elements per thread (mixed)
    std::string err;
};

// An instance prepared on the host (ensc_batch_prepare).
struct ensc_prepared {
    ensc::InstanceHost ih;
    int32_t precision = ENSC_MIXED;
    ensc_material mat{};
};

namespace {

int berr(ensc_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    ensc::set_thread_error(m);
    return code;
}

int bcuda(ensc_batch* b, const char* what, cudaError_t e) {
    return berr(b, e == cudaErrorMemoryAllocation ? ENSC_ERR_OOM : ENSC_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define BCK(b, call)                                      \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) return bcuda((b), #call, _e); \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DevGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

bool is_mixed(const ensc_batch* b) { return b->precision == ENSC_MIXED; }

// Marks the end of the admission work enqueued so far.
int side_mark(ensc_batch* b) {
    BCK(b, cudaEventRecord(b->side_done, b->side));
    b->side_work = true;
    return ENSC_OK;
}

// The batch stream waits for the admission work enqueued so far (no host
// wait); added instances stop being pending.  Every entry point that puts
// work on the batch stream joins first.
int side_join(ensc_batch* b) {
    if (!b->side_work) return ENSC_OK;
    BCK(b, cudaStreamWaitEvent(b->stream, b->side_done, 0));
    b->side_work = false;
    for (Slot& sl : b->inst) sl.pending = false;
    return ENSC_OK;
}

// The stream for a slot's own device work: the admission stream while it is
// pending, else the batch stream (after the cycles already enqueued there).
cudaStream_t slot_stream(const ensc_batch* b, const Slot& sl) { return sl.pending ? b->side : b->stream; }

// Rewrites the instance table and tile lists from the live slots.  The tile
// energy accumulators are folded into the instances first (tile indices
// change) and cleared after.
int rebuild_tables(ensc_batch* b) {
    ensc::launch_between_batch(b->T, b->slots, 1, b->stream);
    BCK(b, cudaGetLastError());
    std::vector<ensc::InstanceDesc> desc(static_cast<size_t>(b->slots));
    std::vector<ensc::NodeView> views(static_cast<size_t>(b->slots));
    std::vector<int32_t> ei, eb, ni, nb;
    std::vector<ensc::ETileSrc> es;
    const int64_t real = is_mixed(b) ? 4 : 8;
    int used_slots = 0;
    for (int s = 0; s < b->slots; ++s) {
        const Slot& sl = b->inst[s];
        ensc::InstanceDesc& d = desc[s];
        d = ensc::InstanceDesc{};
        d.ctl = b->d_ctl + s;
        if (!sl.used) continue;
        used_slots = s + 1;
        d.E = sl.E;
        d.N = sl.N;
        d.M = sl.M;
        // the batched element passes run the J2 update for every instance; an
        // infinite yield stress leaves the elastic update bit-for-bit unchanged
        if (!d.M.plastic) {
            d.M.yield0 = HUGE_VAL;
            d.M.hardening = 0.0;
            ensc::set_mixed_consts(d.M);
        }
        d.active = 1;
        d.patch = sl.PA.pf ? 1 : 0;
        d.pa = sl.PA;
        views[s] = ensc::node_view(d.E, d.N, d.M, d.ctl, &sl.PA);
        d.e_tile0 = static_cast<int32_t>(ei.size());
        for (int64_t e = 0; e < sl.ne; e += b->etile) {
            ei.push_back(s);
            eb.push_back(static_cast<int32_t>(e));
            const ensc::ElemArrays& E = sl.E;
            auto at = [e](const void* p, int64_t size) { return static_cast<const void*>(static_cast<const char*>(p) + e * size); };
            ensc::ETileSrc t{};
            t.conn = at(E.conn, 4);
            t.bt = at(E.bt, real);
            t.vol0 = at(E.vol0, 8);
            t.cbrt_v0 = at(E.cbrt_v0, real);  // mixed: a float copy in the first words
            t.cbrt_v0sq = at(E.cbrt_v0sq, 8);
            t.sigma = at(E.sigma, real);
            t.qia = at(E.qia, real);
            t.eps_p = at(E.eps_p, real);
            t.ne_pad = static_cast<int32_t>(E.ne_pad);
            t.cnt = static_cast<int32_t>(std::min<int64_t>(E.ne_pad - e, b->etile));
            t.slot = s;
            t.base = static_cast<int32_t>(e);
            es.push_back(t);
        }
        d.e_ntiles = static_cast<int32_t>(ei.size()) - d.e_tile0;
        d.n_tile0 = static_cast<int32_t>(ni.size());
        for (int64_t n = 0; n < sl.nn; n += b->ntile) {
            ni.push_back(s);
            nb.push_back(static_cast<int32_t>(n));
        }
        d.n_ntiles = static_cast<int32_t>(ni.size()) - d.n_tile0;
    }
    if (static_cast<int64_t>(ei.size()) > b->max_etiles || static_cast<int64_t>(ni.size()) > b->max_ntiles)
        return berr(b, ENSC_ERR_OOM, "batch tile capacity exceeded");
    const int32_t counts[3] = {static_cast<int32_t>(ei.size()), static_cast<int32_t>(ni.size()), used_slots};
    BCK(b, cudaMemcpyAsync(b->d_desc, desc.data(), desc.size() * sizeof(ensc::InstanceDesc), cudaMemcpyHostToDevice,
                           b->stream));
    BCK(b, cudaMemcpyAsync(b->d_nview, views.data(), views.size() * sizeof(ensc::NodeView), cudaMemcpyHostToDevice,
                           b->stream));
    if (!ei.empty()) {
        BCK(b, cudaMemcpyAsync(b->d_etile_inst, ei.data(), ei.size() * 4, cudaMemcpyHostToDevice, b->stream));
        BCK(b, cudaMemcpyAsync(b->d_etile_base, eb.data(), eb.size() * 4, cudaMemcpyHostToDevice, b->stream));
        BCK(b, cudaMemcpyAsync(b->d_etile_src, es.data(), es.size() * sizeof(ensc::ETileSrc), cudaMemcpyHostToDevice,
                               b->stream));
    }
    if (!ni.empty()) {
        BCK(b, cudaMemcpyAsync(b->d_ntile_inst, ni.data(), ni.size() * 4, cudaMemcpyHostToDevice, b->stream));
        BCK(b, cudaMemcpyAsync(b->d_ntile_base, nb.data(), nb.size() * 4, cudaMemcpyHostToDevice, b->stream));
    }
    BCK(b, cudaMemcpyAsync(b->d_counts, counts, sizeof(counts), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaMemsetAsync(b->d_etile_part, 0, sizeof(double) * 3 * b->max_etiles * (b->etile / 32), b->stream));
    BCK(b, cudaMemsetAsync(b->d_ntile_part, 0, sizeof(double) * 2 * b->max_ntiles, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    b->n_etiles = static_cast<int64_t>(ei.size());
    b->n_ntiles = static_cast<int64_t>(ni.size());
    b->dirty = false;
    return ENSC_OK;
}

void launch_cycle(ensc_batch* b, int ge, int gn, int nt, int ept, cudaStream_t st) {
    ensc::launch_between_batch(b->T, b->slots, 0, st);
    ensc::launch_edge_prepass_batch(b->T, b->sms * b->occ_pre, st);
    if (is_mixed(b)) {
        const bool patch = b->assembly == ENSC_ASSEMBLY_PATCH;
        ensc::launch_element_batch_mixed(b->T, ge, ept, patch, st);
        ensc::launch_node_batch_mixed(b->T, gn, nt, patch, st);
    } else {
        ensc::launch_element_batch_fp64(b->T, ge, st);
        ensc::launch_node_batch_fp64(b->T, gn, nt, st);
    }
}

int occupancy_node(ensc_batch* b, int threads) {
    return std::max(1, is_mixed(b) ? ensc::occupancy_node_batch_mixed(threads)
                                    : ensc::occupancy_node_batch_fp64(threads));
}

int build_graph(ensc_batch* b, const Tune& t) {
    const int nt = t.node_threads;
    const int ge = b->sms * (t.ept == 2 ? b->occ_e2 : b->occ_e) * t.mult_e;
    const int gn = b->sms * occupancy_node(b, nt) * t.mult_n;
    if (b->graph && b->graph_chunk == t.chunk && b->graph_ge == ge && b->graph_gn == gn && b->graph_nt == nt &&
        b->graph_ept == t.ept)
        return ENSC_OK;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    BCK(b, cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    for (int c = 0; c < t.chunk; ++c) launch_cycle(b, ge, gn, nt, t.ept, b->cap_stream);
    cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    if (e != cudaSuccess) return bcuda(b, "cudaStreamEndCapture", e);
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bcuda(b, "cudaGraphInstantiate", e);
    b->graph_chunk = t.chunk;
    b->graph_ge = ge;
    b->graph_gn = gn;
    b->graph_nt = nt;
    b->graph_ept = t.ept;
    return ENSC_OK;
}

// Picks the launch geometry (grid sizes, node-pass block size, elements per
// thread of the mixed element pass) and graph length with the shortest time
// per cycle on the batch as loaded.  The candidates differ only in how work
// is spread over the GPU, not in arithmetic, so the cycles they run are
// ordinary cycles of the solve (the state is identical whichever wins; the
// energy sums are grouped per warp, so with 2 elements per thread they may
// differ in the last bits).  Each candidate runs one warm-up
// graph launch and one timed launch; a run too short for the next candidate
// continues with the best so far, and the next run goes on from there.
constexpr int kTuneCands = 9;
Tune tune_candidate(int i) {
    constexpr int kN = ensc::kNodeThreads;
    const Tune cand[kTuneCands] = {{1, 1, 32, kN, 1},     {2, 1, 32, kN, 1},     {1, 2, 32, kN, 1},
                                   {2, 2, 32, kN, 1},     {1, 1, 32, kN / 2, 1}, {1, 2, 32, kN / 2, 1},
                                   {1, 1, 8, kN, 1},      {1, 1, 32, kN, 2},     {2, 1, 32, kN, 2}};
    return cand[i];
}

// 2 elements per thread: mixed precision, slot assembly (the patch sums take
// one element per thread)
bool candidate_applies(const ensc_batch* b, const Tune& t) {
    return t.ept == 1 || (is_mixed(b) && b->assembly != ENSC_ASSEMBLY_PATCH);
}

int autotune(ensc_batch* b, int64_t* cycles_left) {
    cudaEvent_t e0, e1;
    BCK(b, cudaEventCreate(&e0));
    BCK(b, cudaEventCreate(&e1));
    int rc = ENSC_OK;
    for (; b->tune_next < kTuneCands; ++b->tune_next) {
        Tune t = tune_candidate(b->tune_next);
        if (!candidate_applies(b, t)) continue;
        if (b->fixed_chunk > 0) t.chunk = b->fixed_chunk;
        if (*cycles_left < 2 * t.chunk) break;
        rc = build_graph(b, t);
        if (rc) break;
        cudaError_t e = cudaGraphLaunch(b->graph, b->stream);  // warm-up
        if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(b->graph, b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            rc = bcuda(b, "autotune", e);
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const float per = ms / static_cast<float>(t.chunk);
        if (per < b->tune_best) {
            b->tune_best = per;
            b->tune_pick = t;
        }
        *cycles_left -= 2 * t.chunk;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (b->tune_next == kTuneCands) {
        b->tune = b->tune_pick;
        b->tuned = true;
        b->tunings += 1;
        b->tune_etiles = b->n_etiles;
    } else if (b->tune_best < 1e30f) {
        b->tune = b->tune_pick;
    }
    if (b->fixed_chunk > 0) b->tune.chunk = b->fixed_chunk;
    return build_graph(b, b->tune);
}

// Starts a new tuning when the batch's element tiles have grown or shrunk
// four-fold since the last one (a stream of arrivals and retirements).
void retune_if_reshaped(ensc_batch* b) {
    if (!b->tuned || b->tune_etiles <= 0) return;
    if (b->n_etiles > 4 * b->tune_etiles || 4 * b->n_etiles < b->tune_etiles) {
        b->tuned = false;
        b->tune_next = 0;
        b->tune_best = 1e30f;
    }
}

}  // namespace

extern "C" {

int ensc_batch_create(const ensc_params* params, int32_t max_instances, int64_t max_elements, int64_t max_nodes,
                      int64_t budget_bytes, ensc_batch** out) {
    if (!out || !params) return berr(nullptr, ENSC_ERR_ARG, "params and out are required");
    *out = nullptr;
    if (max_instances <= 0 || max_elements <= 0 || max_nodes <= 0 || budget_bytes <= 0)
        return berr(nullptr, ENSC_ERR_ARG, "batch capacities and budget must be positive");
    if (params->precision != ENSC_FP64 && params->precision != ENSC_MIXED)
        return berr(nullptr, ENSC_ERR_ARG, "unsupported precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || params->device < 0 || params->device >= ndev)
        return berr(nullptr, ENSC_ERR_NODEVICE, "no usable CUDA device");
    ensc_batch* b = new ensc_batch();
    b->device = params->device;
    b->precision = params->precision;
    b->assembly = params->assembly;
    b->budget = budget_bytes;
    b->slots = max_instances;
    // tiles: every instance rounds its element and node counts up to tiles
    b->etile = ensc::batch_element_tile(params->precision == ENSC_MIXED);
    b->ntile = ensc::batch_node_tile(params->precision == ENSC_MIXED);
    b->max_etiles = max_elements / b->etile + max_instances + 1;
    b->max_ntiles = max_nodes / b->ntile + max_instances + 1;
    b->inst.resize(static_cast<size_t>(max_instances));
    if (params->graph_chunk > 0) {
        b->fixed_chunk = static_cast<int>(std::min<int64_t>(params->graph_chunk, 1024));
        b->tune.chunk = b->fixed_chunk;
    }
    DevGuard dg(b->device);
    auto fail = [&](int code) {
        ensc_batch_destroy(b);
        return code;
    };
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, b->device) != cudaSuccess) return fail(berr(b, ENSC_ERR_CUDA, "device query"));
    b->sms = prop.multiProcessorCount;
    b->occ_e = std::max(1, is_mixed(b) ? ensc::occupancy_element_batch_mixed(1) : ensc::occupancy_element_batch_fp64());
    b->occ_e2 = std::max(1, is_mixed(b) ? ensc::occupancy_element_batch_mixed(2) : 1);
    // arena: a memory pool that keeps released blocks for reuse
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = b->device;
    cudaError_t e = cudaMemPoolCreate(&b->pool, &pp);
    if (e != cudaSuccess) return fail(bcuda(b, "cudaMemPoolCreate", e));
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if (params->stream) {
        b->stream = static_cast<cudaStream_t>(params->stream);
    } else {
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(bcuda(b, "cudaStreamCreate", e));
        b->own_stream = true;
    }
    e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(bcuda(b, "cudaStreamCreate", e));
    e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(bcuda(b, "cudaStreamCreate", e));
    e = cudaEventCreateWithFlags(&b->side_done, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(bcuda(b, "cudaEventCreate", e));
    // tables
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t s_desc = al(sizeof(ensc::InstanceDesc) * b->slots), s_et = al(4 * b->max_etiles),
                 s_nt = al(4 * b->max_ntiles), s_cnt = 256, s_ep = al(8 * 3 * b->max_etiles * (b->etile / 32)),
                 s_np = al(8 * 2 * b->max_ntiles), s_ctl = al(sizeof(Ctl) * b->slots),
                 s_scr = al(8 * 3 * static_cast<size_t>(b->scratch_blocks)),
                 s_nprm = al(sizeof(ensc::NodeParam) * b->slots), s_sprm = al(sizeof(ensc::StageHdr) * b->slots),
                 s_esrc = al(sizeof(ensc::ETileSrc) * b->max_etiles), s_nview = al(sizeof(ensc::NodeView) * b->slots);
    const size_t total =
        s_desc + 2 * s_et + 2 * s_nt + s_cnt + s_ep + s_np + s_ctl + s_scr + s_nprm + s_sprm + s_esrc + s_nview;
    e = cudaMalloc(&b->tables, total);
    if (e != cudaSuccess) return fail(bcuda(b, "cudaMalloc(batch tables)", e));
    cudaMemset(b->tables, 0, total);
    char* p = static_cast<char*>(b->tables);
    b->d_desc = reinterpret_cast<ensc::InstanceDesc*>(p);
    p += s_desc;
    b->d_etile_inst = reinterpret_cast<int32_t*>(p);
    p += s_et;
    b->d_etile_base = reinterpret_cast<int32_t*>(p);
    p += s_et;
    b->d_ntile_inst = reinterpret_cast<int32_t*>(p);
    p += s_nt;
    b->d_ntile_base = reinterpret_cast<int32_t*>(p);
    p += s_nt;
    b->d_counts = reinterpret_cast<int32_t*>(p);
    p += s_cnt;
    b->d_etile_part = reinterpret_cast<double*>(p);
    p += s_ep;
    b->d_ntile_part = reinterpret_cast<double*>(p);
    p += s_np;
    b->d_ctl = reinterpret_cast<Ctl*>(p);
    p += s_ctl;
    b->d_scratch = reinterpret_cast<double*>(p);
    p += s_scr;
    b->d_nparam = reinterpret_cast<ensc::NodeParam*>(p);
    p += s_nprm;
    b->d_sparam = reinterpret_cast<ensc::StageHdr*>(p);
    p += s_sprm;
    b->d_etile_src = reinterpret_cast<ensc::ETileSrc*>(p);
    p += s_esrc;
    b->d_nview = reinterpret_cast<ensc::NodeView*>(p);
    e = cudaMallocHost(reinterpret_cast<void**>(&b->h_ctl), sizeof(Ctl) * b->slots);
    if (e != cudaSuccess) return fail(bcuda(b, "cudaMallocHost(ctl)", e));
    std::memset(b->h_ctl, 0, sizeof(Ctl) * b->slots);
    for (int s = 0; s < b->slots; ++s) b->h_ctl[s].done = 1;
    e = cudaMemcpy(b->d_ctl, b->h_ctl, sizeof(Ctl) * b->slots, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(bcuda(b, "ctl init", e));
    b->T.desc = b->d_desc;
    b->T.etile_inst = b->d_etile_inst;
    b->T.etile_base = b->d_etile_base;
    b->T.ntile_inst = b->d_ntile_inst;
    b->T.ntile_base = b->d_ntile_base;
    b->T.counts = b->d_counts;
    b->T.etile_part = b->d_etile_part;
    b->T.ntile_part = b->d_ntile_part;
    b->T.etile = b->etile;
    b->T.ntile = b->ntile;
    b->T.exact_count = b->d_counts + 3;
    b->T.prepass_done = b->d_counts + 4;
    b->T.elem_done = b->d_counts + 5;
    b->T.nparam = b->d_nparam;
    b->T.sparam = b->d_sparam;
    b->T.etile_src = b->d_etile_src;
    b->T.nview = b->d_nview;
    int rc = rebuild_tables(b);
    if (rc) return fail(rc);
    *out = b;
    return ENSC_OK;
}

int ensc_batch_prepare(const ensc_mesh_desc* mesh, const ensc_material* mat, const ensc_params* params,
                       ensc_prepared** out) {
    if (!out) return berr(nullptr, ENSC_ERR_ARG, "out is required");
    *out = nullptr;
    if (!mesh || !mat || !params) return berr(nullptr, ENSC_ERR_ARG, "mesh, material and params are required");
    const int32_t precision = params->precision;
    if (precision != ENSC_FP64 && precision != ENSC_MIXED) return berr(nullptr, ENSC_ERR_ARG, "unknown precision");
    ensc_prepared* p = new (std::nothrow) ensc_prepared;
    if (!p) return berr(nullptr, ENSC_ERR_OOM, "host allocation failed");
    std::string perr;
    int rc;
    try {
        rc = ensc::instance_prepare(mesh, mat, precision == ENSC_MIXED, params->assembly, p->ih, perr);
    } catch (const std::bad_alloc&) {
        rc = ENSC_ERR_OOM;
        perr = "host allocation failed";
    }
    if (rc) {
        delete p;
        return berr(nullptr, rc, perr);
    }
    p->precision = precision;
    p->mat = *mat;
    *out = p;
    return ENSC_OK;
}

int64_t ensc_prepared_bytes(const ensc_prepared* prep) { return prep ? static_cast<int64_t>(prep->ih.bytes) : 0; }

int ensc_prepared_assembly(const ensc_prepared* prep, int32_t* assembly, int64_t* patches, int64_t* partials) {
    if (!prep) return berr(nullptr, ENSC_ERR_ARG, "prep is NULL");
    if (assembly) *assembly = prep->ih.patch ? ENSC_ASSEMBLY_PATCH : ENSC_ASSEMBLY_SLOT;
    if (patches) *patches = prep->ih.n_patches;
    if (partials) *partials = prep->ih.n_pnodes;
    return ENSC_OK;
}

int ensc_prepared_patch_tables(const ensc_prepared* prep, ensc_patch_tables* out) {
    if (!prep || !out) return berr(nullptr, ENSC_ERR_ARG, "prep and out are required");
    const ensc::InstanceHost& h = prep->ih;
    if (!h.patch) return berr(nullptr, ENSC_ERR_ARG, "the instance uses the slot assembly");
    out->n_elements = h.ne;
    out->n_nodes = h.nn;
    out->n_patches = h.n_patches;
    out->n_partials = h.n_pnodes;
    out->stored = h.iperm.data();
    out->patch_first = h.pf_off.data();
    out->inc_first = h.pinc_off.data();
    out->inc = h.pinc.data();
    out->node_first = h.nptr.data();
    out->node_partials = h.nent.data();
    return ENSC_OK;
}

void ensc_prepared_destroy(ensc_prepared* prep) { delete prep; }

int ensc_batch_add(ensc_batch* b, const ensc_mesh_desc* mesh, const ensc_material* mat, const ensc_params* controls,
                   int32_t* slot_out) {
    if (!b || !mesh || !mat || !controls || !slot_out) return berr(b, ENSC_ERR_ARG, "missing argument");
    ensc_prepared* p = nullptr;
    ensc_params pp{};
    pp.precision = b->precision;
    pp.assembly = b->assembly;
    int rc = ensc_batch_prepare(mesh, mat, &pp, &p);
    if (rc) return berr(b, rc, ensc_last_error(nullptr));
    rc = ensc_batch_add_prepared(b, p, controls, slot_out);
    ensc_prepared_destroy(p);
    return rc;
}

int ensc_batch_add_prepared(ensc_batch* b, const ensc_prepared* prep, const ensc_params* controls, int32_t* slot_out) {
    if (!b || !prep || !controls || !slot_out) return berr(b, ENSC_ERR_ARG, "missing argument");
    if (!(controls->factor_timestep > 0.0)) return berr(b, ENSC_ERR_ARG, "factor_timestep must be > 0");
    if (prep->precision != b->precision) return berr(b, ENSC_ERR_ARG, "instance prepared for another precision");
    if (prep->ih.patch != (b->assembly == ENSC_ASSEMBLY_PATCH))
        return berr(b, ENSC_ERR_ARG, "instance prepared for another force assembly");
    DevGuard dg(b->device);
    int s = -1;
    for (int i = 0; i < b->slots; ++i)
        if (!b->inst[i].used) {
            s = i;
            break;
        }
    if (s < 0) return berr(b, ENSC_ERR_OOM, "no free instance slot");
    const ensc::InstanceHost& ih = prep->ih;
    const ensc_material* mat = &prep->mat;
    int rc;
    if (b->used + static_cast<int64_t>(ih.bytes) > b->budget)
        return berr(b, ENSC_ERR_OOM, "instance does not fit the batch's memory budget");
    const int64_t et = (ih.ne + b->etile - 1) / b->etile, nt = (ih.nn + b->ntile - 1) / b->ntile;
    if (b->n_etiles + et > b->max_etiles || b->n_ntiles + nt > b->max_ntiles)
        return berr(b, ENSC_ERR_OOM, "batch tile capacity exceeded");
    Slot& sl = b->inst[s];
    // all on the admission stream: the slot is in no table the batch stream
    // runs until that stream joins it
    cudaStream_t st = b->side;
    void* block = nullptr;
    BCK(b, cudaMallocFromPoolAsync(&block, ih.bytes, b->pool, st));
    std::string perr;
    rc = ensc::instance_upload(ih, block, st, sl.E, sl.N, sl.PA, perr);
    if (rc) {
        cudaFreeAsync(block, st);
        return berr(b, rc, perr);
    }
    sl.block = block;
    sl.bytes = ih.bytes;
    sl.nn = ih.nn;
    sl.ne = ih.ne;
    sl.nn_pad = ih.nn_pad;
    sl.ne_pad = ih.ne_pad;
    sl.plastic = ih.plastic;
    sl.kinetic0_done = false;
    ensc::material_from(mat, controls, sl.M);
    b->h_ctl[s] = ensc::initial_ctl(controls, sl.M);
    b->h_ctl[s].done = 1;  // idle until armed
    // init(): force pass with dt = 0 on the unconstrained velocities
    Ctl c0 = b->h_ctl[s];
    c0.done = 0;
    BCK(b, cudaMemcpyAsync(b->d_ctl + s, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    ensc::Partials P{};
    P.elem = b->d_scratch;
    P.node = b->d_scratch;
    const int g = static_cast<int>(std::min<int64_t>((ih.ne + ensc::kElemThreads - 1) / ensc::kElemThreads,
                                                     b->scratch_blocks));
    P.n_elem_blocks = g;
    if (is_mixed(b)) ensc::launch_element_mixed(sl.E, sl.N, sl.M, b->d_ctl + s, P, g, true, st, sl.PA);
    else ensc::launch_element_fp64(sl.E, sl.N, sl.M, b->d_ctl + s, P, g, true, st);
    BCK(b, cudaGetLastError());
    BCK(b, cudaMemcpyAsync(b->h_ctl + s, b->d_ctl + s, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    BCK(b, cudaStreamSynchronize(st));
    b->h_ctl[s].done = 1;  // idle until armed
    BCK(b, cudaMemcpyAsync(b->d_ctl + s, b->h_ctl + s, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    if (int rcm = side_mark(b)) return rcm;
    sl.pending = true;
    sl.used = true;
    b->used += static_cast<int64_t>(ih.bytes);
    b->dirty = true;  // the tables are rewritten before the next run
    *slot_out = s;
    return ENSC_OK;
}

int ensc_batch_set_bcs(ensc_batch* b, int32_t slot, const int8_t* dof_code, const double* dof_value) {
    if (!b || slot < 0 || slot >= b->slots || !b->inst[slot].used) return berr(b, ENSC_ERR_ARG, "bad slot");
    DevGuard dg(b->device);
    Slot& sl = b->inst[slot];
    cudaStream_t st = slot_stream(b, sl);
    std::vector<uint8_t> bc(static_cast<size_t>(sl.nn_pad), 0);
    std::vector<double> bcv(static_cast<size_t>(3 * sl.nn_pad), 0.0);
    if (dof_code) {
        for (int64_t n = 0; n < sl.nn; ++n) {
            uint32_t packed = 0;
            for (int c = 0; c < 3; ++c) {
                const uint32_t cc = static_cast<uint32_t>(dof_code[3 * n + c]) & 3u;
                packed |= cc << (2 * c);
                if ((cc & ENSC_BC_VELOCITY) && dof_value) bcv[c * sl.nn_pad + n] = dof_value[3 * n + c];
            }
            bc[n] = static_cast<uint8_t>(packed);
        }
    }
    BCK(b, cudaMemcpyAsync(const_cast<uint8_t*>(sl.N.bc), bc.data(), bc.size(), cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(const_cast<double*>(sl.N.bcv), bcv.data(), bcv.size() * 8, cudaMemcpyHostToDevice, st));
    ensc::launch_apply_bc_v(sl.N, is_mixed(b), st);
    if (!sl.kinetic0_done) {
        ensc::Partials P{};
        const int g = static_cast<int>(std::min<int64_t>((sl.nn + ensc::kNodeThreads - 1) / ensc::kNodeThreads,
                                                         b->scratch_blocks));
        P.elem = b->d_scratch;
        P.node = b->d_scratch;
        P.n_elem_blocks = 0;
        P.n_node_blocks = g;
        ensc::launch_kinetic0(sl.N, P, b->d_ctl + slot, is_mixed(b), g, st);
        sl.kinetic0_done = true;
    }
    BCK(b, cudaGetLastError());
    BCK(b, cudaStreamSynchronize(st));
    if (st == b->side) return side_mark(b);
    return ENSC_OK;
}

int ensc_batch_set_gravity_amplitude(ensc_batch* b, int32_t slot, int32_t n_points, const double* time_value) {
    if (!b || slot < 0 || slot >= b->slots || !b->inst[slot].used) return berr(b, ENSC_ERR_ARG, "bad slot");
    if (n_points < 0 || n_points > ENSC_MAX_AMPLITUDE_POINTS || (n_points > 0 && !time_value))
        return berr(b, ENSC_ERR_ARG, "amplitude: 0 to ENSC_MAX_AMPLITUDE_POINTS (time, value) pairs");
    DevGuard dg(b->device);
    if (int rcj = side_join(b)) return rcj;
    Slot& sl = b->inst[slot];
    if (n_points > 0 && !sl.amp)
        BCK(b, cudaMallocFromPoolAsync(reinterpret_cast<void**>(&sl.amp),
                                       2 * sizeof(double) * ENSC_MAX_AMPLITUDE_POINTS, b->pool, b->stream));
    if (n_points > 0) {
        BCK(b, cudaMemcpyAsync(sl.amp, time_value, 2 * sizeof(double) * n_points, cudaMemcpyHostToDevice,
                               b->stream));
        // the caller's table may be pinned memory, which the copy reads in
        // stream order: done before it is handed back
        BCK(b, cudaStreamSynchronize(b->stream));
    }
    sl.M.amp = n_points > 0 ? sl.amp : nullptr;
    sl.M.amp_n = n_points;
    b->dirty = true;  // the instance table carries the material by value
    return ENSC_OK;
}

int ensc_batch_arm(ensc_batch* b, int32_t slot, int64_t max_cycles, double step_end_time) {
    if (!b || slot < 0 || slot >= b->slots || !b->inst[slot].used || max_cycles < 0)
        return berr(b, ENSC_ERR_ARG, "bad slot or cycle count");
    DevGuard dg(b->device);
    cudaStream_t st = slot_stream(b, b->inst[slot]);
    ensc::launch_arm(b->d_ctl + slot, step_end_time, max_cycles, st);
    BCK(b, cudaGetLastError());
    if (st == b->side) return side_mark(b);
    return ENSC_OK;
}

int ensc_batch_run(ensc_batch* b, int64_t cycles) {
    if (!b || cycles < 0) return berr(b, ENSC_ERR_ARG, "bad cycle count");
    if (cycles == 0) return ENSC_OK;
    DevGuard dg(b->device);
    if (int rcj = side_join(b)) return rcj;
    if (b->dirty) {
        int rc = rebuild_tables(b);
        if (rc) return rc;
    }
    retune_if_reshaped(b);
    int64_t left = cycles;
    if (!b->tuned) {
        int rc = autotune(b, &left);
        if (rc) return rc;
    } else {
        int rc = build_graph(b, b->tune);
        if (rc) return rc;
    }
    const int64_t launches = (left + b->tune.chunk - 1) / b->tune.chunk;
    for (int64_t i = 0; i < launches; ++i) BCK(b, cudaGraphLaunch(b->graph, b->stream));
    return ENSC_OK;
}

int ensc_batch_sync(ensc_batch* b, int32_t* n_running) {
    if (!b) return berr(b, ENSC_ERR_ARG, "batch is NULL");
    DevGuard dg(b->device);
    if (int rcj = side_join(b)) return rcj;
    ensc::launch_between_batch(b->T, b->slots, 1, b->stream);  // fold the last cycle's energy
    BCK(b, cudaGetLastError());
    BCK(b, cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(Ctl) * b->slots, cudaMemcpyDeviceToHost, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    int running = 0;
    for (int s = 0; s < b->slots; ++s)
        if (b->inst[s].used && !b->h_ctl[s].done) ++running;
    if (n_running) *n_running = running;
    return ENSC_OK;
}

int ensc_batch_report(ensc_batch* b, int32_t slot, ensc_step_report* r) {
    if (!b || !r || slot < 0 || slot >= b->slots || !b->inst[slot].used) return berr(b, ENSC_ERR_ARG, "bad slot");
    const Ctl& c = b->h_ctl[slot];
    r->time = c.time;
    r->dt_i = c.dt_i;
    r->dt_i_1 = c.dt_i_1;
    r->cycles = c.cycles_done;
    r->total_cycles = c.cycles_done;
    r->status = (c.status & ensc::ST_TIMEOUT) ? ENSC_ERR_TIMEOUT
                : (c.status & ensc::ST_INVERTED) ? ENSC_ERR_INVERTED
                : c.status ? ENSC_ERR_NONFINITE : ENSC_OK;
    r->done = c.done;
    std::memcpy(&r->dt_stable_min, &c.dts_next, sizeof(double));
    return ENSC_OK;
}

int ensc_batch_energy(ensc_batch* b, int32_t slot, ensc_energy_report* out) {
    if (!b || !out || slot < 0 || slot >= b->slots || !b->inst[slot].used) return berr(b, ENSC_ERR_ARG, "bad slot");
    const double* e = b->h_ctl[slot].energy;
    out->kinetic = e[0];
    out->internal = e[1];
    out->hourglass = e[2];
    out->viscous = e[3];
    out->external = e[4];
    out->kinetic0 = e[5];
    return ENSC_OK;
}

int ensc_batch_download(ensc_batch* b, int32_t slot, double* x, double* u, double* v, double* sigma, double* qia,
                        double* eps_p) {
    if (!b || slot < 0 || slot >= b->slots || !b->inst[slot].used) return berr(b, ENSC_ERR_ARG, "bad slot");
    DevGuard dg(b->device);
    if (int rcj = side_join(b)) return rcj;
    const Slot& sl = b->inst[slot];
    const bool mx = is_mixed(b);
    struct Item {
        double* dst;
        const void* src;
        int64_t n, pad;
        int comps;
        bool f32;
        const int32_t* at;
    };
    const int32_t* ep = sl.PA.iperm;  // element fields: stored positions
    const Item items[] = {{x, sl.N.x, sl.nn, sl.nn_pad, 3, false, nullptr},
                          {u, sl.N.u, sl.nn, sl.nn_pad, 3, false, nullptr},
                          {v, sl.N.v, sl.nn, sl.nn_pad, 3, mx, nullptr},
                          {sigma, sl.E.sigma, sl.ne, sl.ne_pad, 6, mx, ep},
                          {qia, sl.E.qia, sl.ne, sl.ne_pad, 12, mx, ep},
                          {eps_p, sl.E.eps_p, sl.ne, sl.ne_pad, 1, mx, ep}};
    const size_t need = static_cast<size_t>(std::max<int64_t>(12 * sl.ne, 3 * sl.nn)) * sizeof(double);
    double* stage = nullptr;
    BCK(b, cudaMallocFromPoolAsync(reinterpret_cast<void**>(&stage), need, b->pool, b->stream));
    int rc = ENSC_OK;
    for (const Item& it : items) {
        if (!it.dst) continue;
        if (it.src == sl.N.v) ensc::launch_v_to_aos(sl.N, mx, stage, b->stream);
        else if (it.src == sl.N.u && mx && ENSC_MIXED_UREF)
            ensc::launch_disp_to_aos(sl.N.x, sl.N.u, sl.nn, sl.nn_pad, stage, b->stream);
        else ensc::launch_soa_to_aos(it.src, it.n, it.pad, it.comps, it.f32, stage, b->stream, it.at);
        cudaError_t e = cudaMemcpyAsync(it.dst, stage, it.n * it.comps * sizeof(double), cudaMemcpyDeviceToHost,
                                        b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) {
            rc = bcuda(b, "batch download", e);
            break;
        }
    }
    cudaFreeAsync(stage, b->stream);
    cudaStreamSynchronize(b->stream);
    return rc;
}

int ensc_batch_remove(ensc_batch* b, int32_t slot) {
    if (!b || slot < 0 || slot >= b->slots || !b->inst[slot].used) return berr(b, ENSC_ERR_ARG, "bad slot");
    DevGuard dg(b->device);
    if (int rcj = side_join(b)) return rcj;
    Slot& sl = b->inst[slot];
    // fold what the instance's tiles still hold (the tables list them until
    // the next run rewrites them), then take it out of the device table so
    // that folds before that rewrite skip the slot, whoever takes it next
    ensc::launch_between_batch(b->T, b->slots, 1, b->stream);
    BCK(b, cudaGetLastError());
    b->h_desc_off = ensc::InstanceDesc{};
    b->h_desc_off.ctl = b->d_ctl + slot;
    BCK(b, cudaMemcpyAsync(b->d_desc + slot, &b->h_desc_off, sizeof(ensc::InstanceDesc), cudaMemcpyHostToDevice,
                           b->stream));
    // the slot idles from now on; its block returns to the pool in stream order
    b->h_ctl[slot] = Ctl{};
    b->h_ctl[slot].done = 1;
    BCK(b, cudaMemcpyAsync(b->d_ctl + slot, b->h_ctl + slot, sizeof(Ctl), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));  // the copies above read host memory
    sl.used = false;
    b->dirty = true;
    const int rc = ENSC_OK;
    if (sl.amp) BCK(b, cudaFreeAsync(sl.amp, b->stream));
    BCK(b, cudaFreeAsync(sl.block, b->stream));
    b->used -= static_cast<int64_t>(sl.bytes);
    sl = Slot{};
    return rc;
}

int64_t ensc_batch_device_bytes(const ensc_batch* b) { return b ? b->used : 0; }

int ensc_batch_tuning(const ensc_batch* b, int32_t* mult_element, int32_t* mult_node, int32_t* graph_cycles,
                      int32_t* node_threads, int32_t* elements_per_thread, int32_t* assembly) {
    if (!b) return ENSC_ERR_ARG;
    const bool t = b->tunings > 0;
    if (mult_element) *mult_element = t ? b->tune.mult_e : 0;
    if (mult_node) *mult_node = t ? b->tune.mult_n : 0;
    if (graph_cycles) *graph_cycles = t ? b->tune.chunk : 0;
    if (node_threads) *node_threads = t ? b->tune.node_threads : 0;
    if (elements_per_thread) *elements_per_thread = t ? b->tune.ept : 0;
    if (assembly) *assembly = b->assembly == ENSC_ASSEMBLY_PATCH ? ENSC_ASSEMBLY_PATCH : ENSC_ASSEMBLY_SLOT;
    return ENSC_OK;
}

int32_t ensc_batch_instances(const ensc_batch* b) {
    if (!b) return 0;
    int n = 0;
    for (const Slot& s : b->inst) n += s.used ? 1 : 0;
    return n;
}

void ensc_batch_destroy(ensc_batch* b) {
    if (!b) return;
    DevGuard dg(b->device);
    if (b->side) cudaStreamSynchronize(b->side);
    side_join(b);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (Slot& s : b->inst) {
        if (s.block) cudaFreeAsync(s.block, b->stream);
        if (s.amp) cudaFreeAsync(s.amp, b->stream);
    }
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->side_done) cudaEventDestroy(b->side_done);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    if (b->pool) cudaMemPoolDestroy(b->pool);
    if (b->tables) cudaFree(b->tables);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    delete b;
}

const char* ensc_batch_last_error(const ensc_batch* b) { return b ? b->err.c_str() : ensc_last_error(nullptr); }

}  // extern "C"
