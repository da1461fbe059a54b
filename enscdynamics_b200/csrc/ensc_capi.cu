// C ABI of the GPU stepper (include/ensc_gpu.h).
//
// Host-side responsibilities, in reference terms:
//   ensc_create   exDyna3D::init() (Explicit3D/source/exDyna3D.cpp:105-142):
//                 element constants and lumped mass (compute_invMassMatrix,
//                 :492-515), the node-to-element gather tables that replace the
//                 8 slot vectors of add_inForce_to_rhs (:523-639), device
//                 allocation, and the init force pass with dt = 0 that seeds
//                 the stable time step.
//   ensc_set_bcs  setCurrentStep's boundary update (:1760-1940, :1911).
//   ensc_step     run()'s loop body (:86-100), as a CUDA graph of cycles.
//   ensc_download copies state back in the reference's array layouts.
#include "ensc_gpu.h"
#include "ensc_device.cuh"
#include "ensc_kernels.h"
#include "ensc_instance.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using ensc::Ctl;

struct ensc_handle {
    int device = 0;
    int precision = ENSC_FP64;
    bool plastic = false;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t cap_stream = nullptr;
    int64_t nn = 0, ne = 0, nn_pad = 0, ne_pad = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    double* staging = nullptr;     // device AoS staging for up/download
    bool staging_owned = false;
    size_t staging_bytes = 0;
    ensc::ElemArrays E{};
    ensc::NodeArrays N{};
    ensc::PatchArrays PA{};        // patch assembly tables (null: slot assembly)
    ensc::Material M{};
    ensc::Partials P{};
    Ctl* ctl = nullptr;            // device
    Ctl* ctl_host = nullptr;       // pinned mirror
    int grid_e = 1, grid_n = 1;
    int chunk = 32;
    cudaGraphExec_t graph = nullptr;
    bool kinetic0_done = false;
    double* amp = nullptr;         // device gravity amplitude table
    // output snapshots (ensc_snapshot_begin / ensc_snapshot_wait): a device
    // buffer of AoS fields and the control block, copied on copy_stream into
    // two pinned host buffers used in turn
    double* snap_dev = nullptr;
    size_t snap_bytes = 0;
    double* snap_host[2] = {nullptr, nullptr};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_captured = nullptr;
    cudaEvent_t snap_landed[2] = {nullptr, nullptr};
    int64_t snap_count = 0;
    bool fe_valid = false;         // fe holds the last force pass's element forces
    int64_t n_patches = 0, n_partials = 0;  // patch assembly
    std::string err;
};

namespace {

thread_local std::string g_create_error;

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

int set_err(ensc_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

int cuda_err(ensc_handle* h, const char* what, cudaError_t e) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return set_err(h, e == cudaErrorMemoryAllocation ? ENSC_ERR_OOM : ENSC_ERR_CUDA, m);
}

#define CK(h, call)                                   \
    do {                                              \
        cudaError_t _e = (call);                      \
        if (_e != cudaSuccess) return cuda_err((h), #call, _e); \
    } while (0)


// Copies a host vector to the device on the handle's stream, so that the
// kernels launched there after it see the data: a plain cudaMemcpy from
// pageable memory may return before its DMA lands, and it is not ordered
// with the handle's non-blocking stream.  (A pageable source is staged
// before the call returns, so the vector may go away after it.)
template <typename T>
int upload(ensc_handle* h, void* dst, const std::vector<T>& src) {
    if (src.empty()) return ENSC_OK;
    CK(h, cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    return ENSC_OK;
}

bool mixed(const ensc_handle* h) { return h->precision == ENSC_MIXED; }

void launch_element(ensc_handle* h, bool init, cudaStream_t st) {
    if (mixed(h)) ensc::launch_element_mixed(h->E, h->N, h->M, h->ctl, h->P, h->grid_e, init, st, h->PA);
    else ensc::launch_element_fp64(h->E, h->N, h->M, h->ctl, h->P, h->grid_e, init, st);
}

void launch_node(ensc_handle* h, cudaStream_t st) {
    if (mixed(h)) ensc::launch_node_mixed(h->E, h->N, h->M, h->ctl, h->P, h->grid_n, st, h->PA);
    else ensc::launch_node_fp64(h->E, h->N, h->M, h->ctl, h->P, h->grid_n, st);
}

int build_graph(ensc_handle* h) {
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(h, cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal));
    for (int c = 0; c < h->chunk; ++c) {
        ensc::launch_between(h->ctl, h->P, 0, h->cap_stream);
        ensc::launch_edge_prepass(h->E, h->N, h->ctl, h->grid_e, h->cap_stream);
        launch_element(h, false, h->cap_stream);
        launch_node(h, h->cap_stream);
    }
    cudaError_t e = cudaStreamEndCapture(h->cap_stream, &g);
    if (e != cudaSuccess) return cuda_err(h, "cudaStreamEndCapture", e);
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_err(h, "cudaGraphInstantiate", e);
    return ENSC_OK;
}

int read_ctl(ensc_handle* h) {
    CK(h, cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return ENSC_OK;
}

int status_code(ensc_handle* h, int32_t st) {
    if (st & ensc::ST_NONFINITE) return set_err(h, ENSC_ERR_NONFINITE, "non-finite nodal state detected");
    if (st & ensc::ST_INVERTED) return set_err(h, ENSC_ERR_INVERTED, "element with J <= 0 detected");
    if (st & ensc::ST_BAD_DT) return set_err(h, ENSC_ERR_NONFINITE, "stable time step is not positive");
    if (st & ensc::ST_TIMEOUT) return set_err(h, ENSC_ERR_TIMEOUT, "a bounded wait for staged element data expired");
    return ENSC_OK;
}

void fill_report(const ensc_handle* h, int64_t before, ensc_step_report* r) {
    if (!r) return;
    const Ctl& c = *h->ctl_host;
    r->time = c.time;
    r->dt_i = c.dt_i;
    r->dt_i_1 = c.dt_i_1;
    r->cycles = c.cycles_done - before;
    r->total_cycles = c.cycles_done;
    r->status = (c.status & ensc::ST_TIMEOUT) ? ENSC_ERR_TIMEOUT
                : (c.status & ensc::ST_INVERTED) ? ENSC_ERR_INVERTED
                : c.status ? ENSC_ERR_NONFINITE : ENSC_OK;
    r->done = c.time < c.step_end ? 0 : 1;
    std::memcpy(&r->dt_stable_min, &c.dts_next, sizeof(double));
}

}  // namespace

namespace ensc {
void set_thread_error(const std::string& msg) { g_create_error = msg; }
}  // namespace ensc

extern "C" {

int ensc_abi_version(void) { return ENSC_ABI_VERSION; }

const char* ensc_last_error(const ensc_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int ensc_create(const ensc_mesh_desc* mesh, const ensc_material* mat, const ensc_params* params,
                ensc_handle** out) {
    if (!out) return set_err(nullptr, ENSC_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!mesh || !mat || !params) return set_err(nullptr, ENSC_ERR_ARG, "mesh, material and params are required");
    if (params->precision != ENSC_FP64 && params->precision != ENSC_MIXED)
        return set_err(nullptr, ENSC_ERR_ARG, "unsupported precision");
    if (!(params->factor_timestep > 0.0)) return set_err(nullptr, ENSC_ERR_ARG, "factor_timestep must be > 0");
    const bool mx = params->precision == ENSC_MIXED;
    ensc::InstanceHost ih;
    std::string perr;
    int rc = ensc::instance_prepare(mesh, mat, mx, params->assembly, ih, perr);
    if (rc) return set_err(nullptr, rc, perr);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= params->device || params->device < 0)
        return set_err(nullptr, ENSC_ERR_NODEVICE, "no usable CUDA device");

    ensc_handle* h = new ensc_handle();
    h->device = params->device;
    h->precision = params->precision;
    h->plastic = ih.plastic;
    h->nn = ih.nn;
    h->ne = ih.ne;
    h->nn_pad = ih.nn_pad;
    h->ne_pad = ih.ne_pad;
    h->chunk = params->graph_chunk > 0 ? params->graph_chunk : 32;
    DevGuard dg(h->device);
    auto fail = [&](int code) {
        g_create_error = h->err;
        ensc_destroy(h);
        return code;
    };

    // ---- launch geometry: persistent grids of (resident blocks per SM) x SMs ----
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) {
        set_err(h, ENSC_ERR_CUDA, "cudaGetDeviceProperties failed");
        return fail(ENSC_ERR_CUDA);
    }
    const int occ_e = std::max(1, mx ? ensc::occupancy_element_mixed(h->plastic) : ensc::occupancy_element_fp64(h->plastic));
    const int occ_n = std::max(1, mx ? ensc::occupancy_node_mixed() : ensc::occupancy_node_fp64());
    const int64_t ge = (h->ne + ensc::kElemThreads - 1) / ensc::kElemThreads;
    const int64_t node_threads = static_cast<int64_t>(ensc::kNodeThreads) * ensc::node_group_width(mx);
    const int64_t gn = (h->nn + node_threads - 1) / node_threads;
    h->grid_e = static_cast<int>(std::min<int64_t>(ge, static_cast<int64_t>(occ_e) * prop.multiProcessorCount));
    h->grid_n = static_cast<int>(std::min<int64_t>(gn, static_cast<int64_t>(occ_n) * prop.multiProcessorCount));

    // ---- device memory: the instance block plus partial sums and control ----
    const size_t pbytes = (3 * static_cast<size_t>(h->grid_e) + 2 * static_cast<size_t>(h->grid_n)) * sizeof(double);
    const size_t small = (pbytes + 255) / 256 * 256 + (sizeof(Ctl) + 255) / 256 * 256;
    cudaError_t ce = cudaMalloc(&h->arena, ih.bytes + small);
    if (ce != cudaSuccess) {
        cuda_err(h, "cudaMalloc(instance)", ce);
        return fail(ENSC_ERR_OOM);
    }
    h->arena_bytes = ih.bytes + small;
    if (cudaMallocHost(reinterpret_cast<void**>(&h->ctl_host), sizeof(Ctl)) != cudaSuccess) {
        set_err(h, ENSC_ERR_OOM, "cudaMallocHost(ctl)");
        return fail(ENSC_ERR_OOM);
    }
    if (params->stream) {
        h->stream = static_cast<cudaStream_t>(params->stream);
    } else {
        ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) {
            cuda_err(h, "cudaStreamCreate", ce);
            return fail(ENSC_ERR_CUDA);
        }
        h->own_stream = true;
    }
    ce = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        cuda_err(h, "cudaStreamCreate(capture)", ce);
        return fail(ENSC_ERR_CUDA);
    }
    rc = ensc::instance_upload(ih, h->arena, h->stream, h->E, h->N, h->PA, perr);
    if (rc) {
        set_err(h, rc, perr);
        return fail(rc);
    }
    h->n_patches = ih.n_patches;
    h->n_partials = ih.n_pnodes;
    char* tail = static_cast<char*>(h->arena) + ih.bytes;
    h->P.elem = reinterpret_cast<double*>(tail);
    h->P.node = h->P.elem + 3 * h->grid_e;
    h->P.n_elem_blocks = h->grid_e;
    h->P.n_node_blocks = h->grid_n;
    h->ctl = reinterpret_cast<Ctl*>(tail + (pbytes + 255) / 256 * 256);
    ce = cudaMemsetAsync(tail, 0, small, h->stream);
    if (ce != cudaSuccess) {
        cuda_err(h, "cudaMemset(partials)", ce);
        return fail(ENSC_ERR_CUDA);
    }
    // staging for AoS up/download: reuse the element force scratch when large enough
    const size_t need_stage = std::max<size_t>(12 * h->ne, 3 * h->nn) * sizeof(double);
    if (ih.size[ensc::InstanceHost::FE] >= need_stage) {
        h->staging = static_cast<double*>(h->E.fe);
    } else {
        ce = cudaMalloc(reinterpret_cast<void**>(&h->staging), need_stage);
        if (ce != cudaSuccess) {
            cuda_err(h, "cudaMalloc(staging)", ce);
            return fail(ENSC_ERR_OOM);
        }
        h->staging_owned = true;
    }
    h->staging_bytes = need_stage;

    ensc::material_from(mat, params, h->M);
    *h->ctl_host = ensc::initial_ctl(params, h->M);
    ce = cudaMemcpyAsync(h->ctl, h->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream);
    if (ce != cudaSuccess) {
        cuda_err(h, "upload ctl", ce);
        return fail(ENSC_ERR_CUDA);
    }
    // init(): the force pass with dt = 0 and no boundary conditions, which
    // leaves the minimum element dt for the first cycle in ctl->dts_next
    launch_element(h, true, h->stream);
    ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) {
        cuda_err(h, "init pass", ce);
        return fail(ENSC_ERR_CUDA);
    }
    rc = build_graph(h);
    if (rc) return fail(rc);
    *out = h;
    return ENSC_OK;
}

int ensc_set_bcs(ensc_handle* h, const int8_t* dof_code, const double* dof_value) {
    if (!h) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    std::vector<uint8_t> bc(static_cast<size_t>(h->nn_pad), 0);
    std::vector<double> bcv(static_cast<size_t>(3 * h->nn_pad), 0.0);
    if (dof_code) {
        for (int64_t n = 0; n < h->nn; ++n) {
            uint32_t packed = 0;
            for (int c = 0; c < 3; ++c) {
                const uint32_t cc = static_cast<uint32_t>(dof_code[3 * n + c]) & 3u;
                packed |= cc << (2 * c);
                if ((cc & ENSC_BC_VELOCITY) && dof_value) bcv[c * h->nn_pad + n] = dof_value[3 * n + c];
            }
            bc[n] = static_cast<uint8_t>(packed);
        }
    }
    int rc = upload(h, const_cast<uint8_t*>(h->N.bc), bc);
    if (!rc) rc = upload(h, const_cast<double*>(h->N.bcv), bcv);
    if (rc) return rc;
    ensc::launch_apply_bc_v(h->N, mixed(h), h->stream);
    if (!h->kinetic0_done) {
        ensc::launch_kinetic0(h->N, h->P, h->ctl, mixed(h), h->grid_n, h->stream);
        h->kinetic0_done = true;
    }
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->stream));
    return ENSC_OK;
}

int ensc_set_gravity(ensc_handle* h, int32_t on, double value, const double dir[3]) {
    if (!h) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    h->M.gravity_on = on;
    h->M.gravity_value = value;
    for (int i = 0; i < 3; ++i) h->M.gravity_dir[i] = dir ? dir[i] : 0.0;
    return build_graph(h);
}

int ensc_set_gravity_amplitude(ensc_handle* h, int32_t n_points, const double* time_value) {
    if (!h) return ENSC_ERR_ARG;
    if (n_points < 0 || n_points > ENSC_MAX_AMPLITUDE_POINTS || (n_points > 0 && !time_value))
        return set_err(h, ENSC_ERR_ARG, "amplitude: 0 to ENSC_MAX_AMPLITUDE_POINTS (time, value) pairs");
    DevGuard dg(h->device);
    if (n_points == 0) {
        h->M.amp = nullptr;
        h->M.amp_n = 0;
        return build_graph(h);
    }
    if (!h->amp) {
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&h->amp), 2 * sizeof(double) * ENSC_MAX_AMPLITUDE_POINTS);
        if (e != cudaSuccess) {
            h->amp = nullptr;
            return cuda_err(h, "cudaMalloc(amplitude)", e);
        }
    }
    // stream order: cycles already enqueued finish with the previous table
    CK(h, cudaMemcpyAsync(h->amp, time_value, 2 * sizeof(double) * n_points, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    h->M.amp = h->amp;
    h->M.amp_n = n_points;
    return build_graph(h);
}

int ensc_step_async(ensc_handle* h, int64_t max_cycles, double step_end_time) {
    if (!h || max_cycles < 0) return ENSC_ERR_ARG;
    if (max_cycles == 0) return ENSC_OK;
    DevGuard dg(h->device);
    ensc::launch_arm(h->ctl, step_end_time, max_cycles, h->stream);
    const int64_t launches = (max_cycles + h->chunk - 1) / h->chunk;
    for (int64_t i = 0; i < launches; ++i) CK(h, cudaGraphLaunch(h->graph, h->stream));
    CK(h, cudaGetLastError());
    h->fe_valid = true;
    return ENSC_OK;
}

int ensc_step_until_async(ensc_handle* h, int64_t max_cycles, double step_end_time, double pause_time) {
    if (!h || max_cycles < 0) return ENSC_ERR_ARG;
    if (max_cycles > (int64_t(1) << 24))
        return set_err(h, ENSC_ERR_ARG, "ensc_step_until_async: at most 2^24 cycles per call");
    if (max_cycles == 0) return ENSC_OK;
    DevGuard dg(h->device);
    ensc::launch_arm(h->ctl, step_end_time, max_cycles, h->stream, pause_time);
    const int64_t launches = (max_cycles + h->chunk - 1) / h->chunk;
    for (int64_t i = 0; i < launches; ++i) CK(h, cudaGraphLaunch(h->graph, h->stream));
    CK(h, cudaGetLastError());
    h->fe_valid = true;
    return ENSC_OK;
}

int ensc_sync(ensc_handle* h, ensc_step_report* report) {
    if (!h) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    const int64_t before = h->ctl_host->cycles_done;
    ensc::launch_between(h->ctl, h->P, 1, h->stream);
    CK(h, cudaGetLastError());
    int rc = read_ctl(h);
    if (rc) return rc;
    fill_report(h, before, report);
    return status_code(h, h->ctl_host->status);
}

int ensc_step(ensc_handle* h, int64_t max_cycles, double step_end_time, ensc_step_report* report) {
    return ensc_step_until(h, max_cycles, step_end_time, HUGE_VAL, report);
}

int ensc_step_until(ensc_handle* h, int64_t max_cycles, double step_end_time, double pause_time,
                    ensc_step_report* report) {
    if (!h || max_cycles < 0) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    const int64_t before = h->ctl_host->cycles_done;
    if (max_cycles > 0) {
        ensc::launch_arm(h->ctl, step_end_time, max_cycles, h->stream, pause_time);
        // launch graphs in batches; between batches read the control block
        // to stop once time reached step_end
        const int64_t batch = std::max<int64_t>(1, 4096 / h->chunk);
        int64_t launched = 0;
        const int64_t needed = (max_cycles + h->chunk - 1) / h->chunk;
        while (launched < needed) {
            const int64_t n = std::min(batch, needed - launched);
            for (int64_t i = 0; i < n; ++i) CK(h, cudaGraphLaunch(h->graph, h->stream));
            launched += n;
            h->fe_valid = true;
            int rc = read_ctl(h);
            if (rc) return rc;
            if (h->ctl_host->done || h->ctl_host->status) break;
        }
    }
    ensc::launch_between(h->ctl, h->P, 1, h->stream);
    CK(h, cudaGetLastError());
    int rc = read_ctl(h);
    if (rc) return rc;
    fill_report(h, before, report);
    return status_code(h, h->ctl_host->status);
}

// The staging area may be the element force scratch, whose slots no
// element fills must read as zeros for the node pass: clear what was used.
static int release_staging(ensc_handle* h, size_t used) {
    if (!h->staging_owned && used) {
        h->fe_valid = false;
        CK(h, cudaMemsetAsync(h->staging, 0, used, h->stream));
    }
    return ENSC_OK;
}

int ensc_download(ensc_handle* h, double* x, double* u, double* v, double* sigma, double* qia, double* eps_p) {
    if (!h) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    struct Item {
        double* dst;
        const void* src;
        int64_t n, pad;
        int comps;
        bool f32;
        const int32_t* at;
    };
    const bool mx = mixed(h);
    const int32_t* ep = h->PA.iperm;  // element fields: stored positions
    const Item items[] = {{x, h->N.x, h->nn, h->nn_pad, 3, false, nullptr},
                          {u, h->N.u, h->nn, h->nn_pad, 3, false, nullptr},
                          {v, h->N.v, h->nn, h->nn_pad, 3, mx, nullptr},
                          {sigma, h->E.sigma, h->ne, h->ne_pad, 6, mx, ep},
                          {qia, h->E.qia, h->ne, h->ne_pad, 12, mx, ep},
                          {eps_p, h->E.eps_p, h->ne, h->ne_pad, 1, mx, ep}};
    size_t used = 0;
    for (const Item& it : items) {
        if (!it.dst) continue;
        if (it.src == h->N.v) ensc::launch_v_to_aos(h->N, mx, h->staging, h->stream);
        else if (it.src == h->N.u && mx && ENSC_MIXED_UREF)
            ensc::launch_disp_to_aos(h->N.x, h->N.u, h->nn, h->nn_pad, h->staging, h->stream);
        else ensc::launch_soa_to_aos(it.src, it.n, it.pad, it.comps, it.f32, h->staging, h->stream, it.at);
        CK(h, cudaGetLastError());
        CK(h, cudaMemcpyAsync(it.dst, h->staging, it.n * it.comps * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        used = std::max(used, static_cast<size_t>(it.n * it.comps) * sizeof(double));
    }
    return release_staging(h, used);
}

int ensc_download_reactions(ensc_handle* h, double* rf) {
    if (!h || !rf) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    ensc::launch_soa_to_aos(h->N.rf, h->nn, h->nn_pad, 3, false, h->staging, h->stream);
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(rf, h->staging, h->nn * 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return release_staging(h, static_cast<size_t>(h->nn * 3) * sizeof(double));
}

int ensc_upload_state(ensc_handle* h, const double* x, const double* u, const double* v, const double* sigma,
                      const double* qia, const double* eps_p, double time, double dt_i, double dt_i_1,
                      double dt_stable_min) {
    if (!h) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    struct Item {
        const double* src;
        void* dst;
        int64_t n, pad;
        int comps;
        bool f32;
        const int32_t* at;
    };
    const bool mx = mixed(h);
    const int32_t* ep = h->PA.iperm;  // element fields: stored positions
    const Item items[] = {{x, h->N.x, h->nn, h->nn_pad, 3, false, nullptr},
                          {u, h->N.u, h->nn, h->nn_pad, 3, false, nullptr},
                          {v, h->N.v, h->nn, h->nn_pad, 3, mx, nullptr},
                          {sigma, h->E.sigma, h->ne, h->ne_pad, 6, mx, ep},
                          {qia, h->E.qia, h->ne, h->ne_pad, 12, mx, ep},
                          {eps_p, h->E.eps_p, h->ne, h->ne_pad, 1, mx, ep}};
    size_t used = 0;
    // mixed: the u rows hold x - u; they hold u while x and u are replaced
    const bool uref = mx && ENSC_MIXED_UREF && (x || u);
    if (uref) ensc::launch_reflect_rows(h->N.x, h->N.u, h->nn, h->nn_pad, h->stream);
    cudaError_t ue = cudaGetLastError();
    const char* what = "ensc_upload_state";
    for (const Item& it : items) {
        if (!it.src || ue != cudaSuccess) continue;
        ue = cudaMemcpyAsync(h->staging, it.src, it.n * it.comps * sizeof(double), cudaMemcpyHostToDevice,
                             h->stream);
        if (ue != cudaSuccess) {
            what = "cudaMemcpyAsync(state upload)";
            break;
        }
        if (it.dst == h->N.v) ensc::launch_aos_to_v(h->staging, h->N, mx, h->stream);
        else ensc::launch_aos_to_soa(h->staging, it.n, it.pad, it.comps, it.dst, it.f32, h->stream, it.at);
        ue = cudaGetLastError();
        used = std::max(used, static_cast<size_t>(it.n * it.comps) * sizeof(double));
    }
    // back to x - u in the u rows, also when an upload above failed
    if (uref) ensc::launch_reflect_rows(h->N.x, h->N.u, h->nn, h->nn_pad, h->stream);
    if (ue == cudaSuccess) ue = cudaGetLastError();
    if (ue != cudaSuccess) {
        release_staging(h, used);
        return cuda_err(h, what, ue);
    }
    if (int rc0 = release_staging(h, used)) return rc0;
    int rc = read_ctl(h);
    if (rc) return rc;
    h->ctl_host->time = time;
    h->ctl_host->dt_i = dt_i;
    h->ctl_host->dt_i_1 = dt_i_1;
    if (dt_stable_min > 0.0) {
        long long b;
        std::memcpy(&b, &dt_stable_min, sizeof b);
        h->ctl_host->dts_next = static_cast<unsigned long long>(b);
    }
    CK(h, cudaMemcpyAsync(h->ctl, h->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return ENSC_OK;
}

int ensc_snapshot_begin(ensc_handle* h) {
    if (!h) return ENSC_ERR_ARG;
    if (!h->fe_valid)
        return set_err(h, ENSC_ERR_ARG,
                       "ensc_snapshot_begin: no force pass since the last download or upload; run a cycle first");
    DevGuard dg(h->device);
    const size_t nodes3 = static_cast<size_t>(3 * h->nn), elems6 = static_cast<size_t>(6 * h->ne);
    const size_t fields = (5 * nodes3 + elems6) * sizeof(double);
    if (!h->snap_dev) {
        h->snap_bytes = (fields + 255) / 256 * 256 + sizeof(Ctl);
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&h->snap_dev), h->snap_bytes);
        if (e != cudaSuccess) {
            h->snap_dev = nullptr;
            return cuda_err(h, "cudaMalloc(snapshot)", e);
        }
        for (int k = 0; k < 2; ++k) {
            e = cudaMallocHost(reinterpret_cast<void**>(&h->snap_host[k]), h->snap_bytes);
            if (e != cudaSuccess) {
                h->snap_host[k] = nullptr;
                return cuda_err(h, "cudaMallocHost(snapshot)", e);
            }
        }
        CK(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
        CK(h, cudaEventCreateWithFlags(&h->snap_captured, cudaEventDisableTiming));
        for (int k = 0; k < 2; ++k) CK(h, cudaEventCreateWithFlags(&h->snap_landed[k], cudaEventDisableTiming));
    }
    // the previous snapshot's copy to the host reads the device buffer this
    // one overwrites (the copy before it used the same host buffer and ran
    // earlier on the same copy stream)
    if (h->snap_count > 0) CK(h, cudaStreamWaitEvent(h->stream, h->snap_landed[(h->snap_count - 1) % 2], 0));
    double* d = h->snap_dev;
    const bool mx = mixed(h);
    if (mx) ensc::launch_acceleration_mixed(h->E, h->N, h->M, h->ctl, d + 3 * nodes3, h->stream, h->PA);
    else ensc::launch_acceleration_fp64(h->E, h->N, h->M, h->ctl, d + 3 * nodes3, h->stream);
    ensc::launch_soa_to_aos(h->N.x, h->nn, h->nn_pad, 3, false, d, h->stream);
    if (mx && ENSC_MIXED_UREF) ensc::launch_disp_to_aos(h->N.x, h->N.u, h->nn, h->nn_pad, d + nodes3, h->stream);
    else ensc::launch_soa_to_aos(h->N.u, h->nn, h->nn_pad, 3, false, d + nodes3, h->stream);
    ensc::launch_v_to_aos(h->N, mx, d + 2 * nodes3, h->stream);
    ensc::launch_soa_to_aos(h->N.rf, h->nn, h->nn_pad, 3, false, d + 4 * nodes3, h->stream);
    ensc::launch_soa_to_aos(h->E.sigma, h->ne, h->ne_pad, 6, mx, d + 5 * nodes3, h->stream, h->PA.iperm);
    CK(h, cudaGetLastError());
    char* ctl_copy = reinterpret_cast<char*>(d) + (h->snap_bytes - sizeof(Ctl));
    CK(h, cudaMemcpyAsync(ctl_copy, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToDevice, h->stream));
    CK(h, cudaEventRecord(h->snap_captured, h->stream));
    const int k = static_cast<int>(h->snap_count % 2);
    CK(h, cudaStreamWaitEvent(h->copy_stream, h->snap_captured, 0));
    CK(h, cudaMemcpyAsync(h->snap_host[k], h->snap_dev, h->snap_bytes, cudaMemcpyDeviceToHost, h->copy_stream));
    CK(h, cudaEventRecord(h->snap_landed[k], h->copy_stream));
    h->snap_count += 1;
    return ENSC_OK;
}

int ensc_snapshot_wait(ensc_handle* h, ensc_snapshot* out) {
    if (!h || !out) return ENSC_ERR_ARG;
    if (h->snap_count == 0) return set_err(h, ENSC_ERR_ARG, "ensc_snapshot_wait: no snapshot begun");
    DevGuard dg(h->device);
    const int k = static_cast<int>((h->snap_count - 1) % 2);
    CK(h, cudaEventSynchronize(h->snap_landed[k]));
    const double* b = h->snap_host[k];
    const size_t nodes3 = static_cast<size_t>(3 * h->nn);
    out->x = b;
    out->u = b + nodes3;
    out->v = b + 2 * nodes3;
    out->a = b + 3 * nodes3;
    out->rf = b + 4 * nodes3;
    out->sigma = b + 5 * nodes3;
    Ctl c;
    std::memcpy(&c, reinterpret_cast<const char*>(b) + (h->snap_bytes - sizeof(Ctl)), sizeof(Ctl));
    out->time = c.time;
    out->dt_i = c.dt_i;
    out->dt_i_1 = c.dt_i_1;
    out->total_cycles = c.cycles_done;
    out->status = (c.status & ensc::ST_TIMEOUT) ? ENSC_ERR_TIMEOUT
                  : (c.status & ensc::ST_INVERTED) ? ENSC_ERR_INVERTED
                  : c.status ? ENSC_ERR_NONFINITE : ENSC_OK;
    return ENSC_OK;
}

int ensc_energy(ensc_handle* h, ensc_energy_report* out) {
    if (!h || !out) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    ensc::launch_between(h->ctl, h->P, 1, h->stream);
    CK(h, cudaGetLastError());
    int rc = read_ctl(h);
    if (rc) return rc;
    const double* e = h->ctl_host->energy;
    out->kinetic = e[0];
    out->internal = e[1];
    out->hourglass = e[2];
    out->viscous = e[3];
    out->external = e[4];
    out->kinetic0 = e[5];
    return ENSC_OK;
}

int ensc_profile(ensc_handle* h, int64_t max_cycles, double step_end_time, double ms[5], int64_t launches[5]) {
    if (!h || max_cycles < 0 || !ms || !launches) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    for (int i = 0; i < 5; ++i) {
        ms[i] = 0.0;
        launches[i] = 0;
    }
    cudaEvent_t ev[6];
    for (int i = 0; i < 6; ++i) CK(h, cudaEventCreate(&ev[i]));
    ensc::launch_arm(h->ctl, step_end_time, max_cycles, h->stream);
    int rc = ENSC_OK;
    for (int64_t c = 0; c < max_cycles && rc == ENSC_OK; ++c) {
        cudaEventRecord(ev[0], h->stream);
        ensc::launch_between(h->ctl, h->P, 0, h->stream);
        cudaEventRecord(ev[1], h->stream);
        ensc::launch_edge_prepass(h->E, h->N, h->ctl, h->grid_e, h->stream);
        cudaEventRecord(ev[2], h->stream);
        cudaEventRecord(ev[3], h->stream);  // begin_exact runs inside the prepass
        launch_element(h, false, h->stream);
        cudaEventRecord(ev[4], h->stream);
        launch_node(h, h->stream);
        cudaEventRecord(ev[5], h->stream);
        cudaError_t e = cudaEventSynchronize(ev[5]);
        if (e != cudaSuccess) {
            rc = cuda_err(h, "ensc_profile", e);
            break;
        }
        for (int k = 0; k < 5; ++k) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms[k] += t;
            launches[k] += 1;
        }
        if (read_ctl(h) != ENSC_OK) break;
        if (h->ctl_host->done) break;
    }
    for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
    return rc;
}

int64_t ensc_device_bytes(const ensc_handle* h) {
    if (!h) return 0;
    return static_cast<int64_t>(h->arena_bytes + (h->staging_owned ? h->staging_bytes : 0));
}

int32_t ensc_kernels_per_cycle(const ensc_handle* h) { return h ? 4 : 0; }

int ensc_assembly(const ensc_handle* h, int32_t* assembly, int64_t* patches, int64_t* partials) {
    if (!h) return ENSC_ERR_ARG;
    if (assembly) *assembly = h->PA.pf ? ENSC_ASSEMBLY_PATCH : ENSC_ASSEMBLY_SLOT;
    if (patches) *patches = h->n_patches;
    if (partials) *partials = h->n_partials;
    return ENSC_OK;
}

void ensc_destroy(ensc_handle* h) {
    if (!h) return;
    DevGuard dg(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    if (h->staging_owned && h->staging) cudaFree(h->staging);
    if (h->arena) cudaFree(h->arena);
    if (h->amp) cudaFree(h->amp);
    if (h->copy_stream) {
        cudaStreamSynchronize(h->copy_stream);
        cudaStreamDestroy(h->copy_stream);
    }
    if (h->snap_captured) cudaEventDestroy(h->snap_captured);
    for (int k = 0; k < 2; ++k) {
        if (h->snap_landed[k]) cudaEventDestroy(h->snap_landed[k]);
        if (h->snap_host[k]) cudaFreeHost(h->snap_host[k]);
    }
    if (h->snap_dev) cudaFree(h->snap_dev);
    if (h->ctl_host) cudaFreeHost(h->ctl_host);
    delete h;
}

}  // extern "C"
