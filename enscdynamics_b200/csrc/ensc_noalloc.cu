// ensc_step_noalloc: the FP64 stepper for callers that cannot allocate
// device memory.
//
// Some hosts of this stepper may not call cudaMalloc: plug-ins of an
// application that owns and pre-plans all device memory through its own
// pool (the application accounts for every byte and an allocation behind
// its back can fail its budget or fragment its pool), and solver loops with
// a memory budget fixed at start-up (cudaMalloc can synchronise the device
// and its failure mid-run cannot be handled there).  They can hand over
// device arrays they already own for the model and its state, but they
// cannot provide the stepper's internal scratch.  This entry point keeps
// that scratch -- the per-element force hand-off between the element pass
// and the node gather, the per-block energy partials and the control block --
// in one file-scope __device__ array of fixed size, so a call performs no
// allocation at all.
//
// Limits and sharing:
//   * at most ENSC_NOALLOC_MAX_ELEMENTS elements and ENSC_NOALLOC_MAX_NODES
//     nodes per call; larger meshes are rejected with ENSC_ERR_ARG;
//   * every GPU that loads this library holds the array (about 6.3 MiB) until
//     the process exits;
//   * all calls share the one array per device and it keeps the last call's
//     contents; each call re-initialises what must start from zero or +inf,
//     but two calls that overlap on the GPU (different streams or host
//     threads at the same time) race on it and corrupt each other;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     that first call before any stream capture;
//   * the call launches its cycles in batches of kBatchCycles and reads the
//     control block back after each batch (it waits for the stream), so it
//     returns as soon as the step end or a status stops the run, whatever
//     max_cycles is.
#include "ensc_gpu.h"
#include "ensc_device.cuh"
#include "ensc_kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

namespace {

constexpr int kMaxDevices = 64;
// cycles launched between two read-backs of the control block
constexpr int64_t kBatchCycles = 32;
constexpr int kMaxElemBlocks = (ENSC_NOALLOC_MAX_ELEMENTS + ensc::kElemThreads - 1) / ensc::kElemThreads;
constexpr int kMaxNodeBlocks = (ENSC_NOALLOC_MAX_NODES + ensc::kNodeThreads - 1) / ensc::kNodeThreads;
constexpr size_t kCtlBytes = (sizeof(ensc::Ctl) + 255) / 256 * 256;
constexpr size_t kPartialBytes = ((3 * kMaxElemBlocks + 2 * kMaxNodeBlocks) * sizeof(double) + 255) / 256 * 256;
constexpr size_t kForceBytes = size_t(24) * ENSC_NOALLOC_MAX_ELEMENTS * sizeof(double);
constexpr size_t kScratchBytes = kCtlBytes + kPartialBytes + kForceBytes;

// The scratch: [control block][energy partials][element forces 24 x ne].
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// messages are reported through ensc_last_error(NULL), like ensc_create's
int fail(int code, const std::string& msg) {
    ensc::set_thread_error(msg);
    return code;
}

// Device address of the scratch on `dev`, looked up once per device with
// that device current.
int scratch_address(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(ENSC_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_addr[dev]);
    return ENSC_OK;
}

}  // namespace

extern "C" {

int ensc_step_noalloc(const ensc_device_model* m, const ensc_material* mat, const ensc_params* params,
                      ensc_noalloc_clock* clk, int64_t max_cycles, double step_end_time) {
    if (!m || !mat || !params || !clk || max_cycles < 0) return fail(ENSC_ERR_ARG, "missing argument");
    if (m->n_elements <= 0 || m->n_nodes <= 0) return fail(ENSC_ERR_ARG, "empty mesh");
    if (m->n_elements > ENSC_NOALLOC_MAX_ELEMENTS || m->n_nodes > ENSC_NOALLOC_MAX_NODES)
        return fail(ENSC_ERR_ARG, "mesh exceeds the no-allocation limits (ENSC_NOALLOC_MAX_ELEMENTS = " +
                                      std::to_string(ENSC_NOALLOC_MAX_ELEMENTS) + ", ENSC_NOALLOC_MAX_NODES = " +
                                      std::to_string(ENSC_NOALLOC_MAX_NODES) + ")");
    if (params->precision != ENSC_FP64) return fail(ENSC_ERR_ARG, "the no-allocation stepper is FP64 only");
    if (!m->conn || !m->bt || !m->vol0 || !m->cbrt_v0 || !m->cbrt_v0sq || !m->inv_mass || !m->bc ||
        !m->bc_value || !m->node_elem || !m->x || !m->u || !m->v || !m->sigma || !m->qia || !m->eps_p || !m->rf)
        return fail(ENSC_ERR_ARG, "a device array of the model is NULL");
    if (params->device < 0 || params->device >= kMaxDevices) return fail(ENSC_ERR_ARG, "bad device ordinal");
    if (!(mat->rho > 0.0) || !(mat->E > 0.0) || !(mat->nu < 0.5)) return fail(ENSC_ERR_ARG, "invalid material");
    if (m->gravity_amp_n < 0 || m->gravity_amp_n > ENSC_MAX_AMPLITUDE_POINTS ||
        (m->gravity_amp_n > 0 && !m->gravity_amp))
        return fail(ENSC_ERR_ARG, "bad gravity amplitude table");

    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != params->device && cudaSetDevice(params->device) != cudaSuccess)
        return fail(ENSC_ERR_NODEVICE, "cannot select the device");
    struct Restore {
        int d;
        ~Restore() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{prev != params->device ? prev : -1};

    unsigned char* base = nullptr;
    int rc = scratch_address(params->device, &base);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(params->stream);
    const int64_t ne = m->n_elements, nn = m->n_nodes;

    ensc::Ctl* ctl = reinterpret_cast<ensc::Ctl*>(base);
    ensc::Partials P{};
    P.n_elem_blocks = static_cast<int32_t>((ne + ensc::kElemThreads - 1) / ensc::kElemThreads);
    P.n_node_blocks = static_cast<int32_t>((nn + ensc::kNodeThreads - 1) / ensc::kNodeThreads);
    P.elem = reinterpret_cast<double*>(base + kCtlBytes);
    P.node = P.elem + 3 * kMaxElemBlocks;
    double* fe = reinterpret_cast<double*>(base + kCtlBytes + kPartialBytes);

    ensc::ElemArrays E{};
    E.ne = ne;
    E.ne_pad = ne;
    E.conn = m->conn;
    E.bt = m->bt;
    E.vol0 = m->vol0;
    E.cbrt_v0 = m->cbrt_v0;
    E.cbrt_v0sq = m->cbrt_v0sq;
    E.sigma = m->sigma;
    E.qia = m->qia;
    E.eps_p = m->eps_p;
    E.fe = fe;
    ensc::NodeArrays N{};
    N.nn = nn;
    N.nn_pad = nn;
    N.x = m->x;
    N.u = m->u;
    N.v = m->v;
    N.inv_mass = m->inv_mass;
    N.bc = m->bc;
    N.bcv = m->bc_value;
    N.ell = m->node_elem;
    N.csr_ptr = nullptr;
    N.csr_ent = nullptr;
    N.rf = m->rf;

    ensc::Material M{};
    M.E = mat->E;
    M.nu = mat->nu;
    M.rho = mat->rho;
    M.G = M.E / ((1.0 + M.nu) * 2.0);
    M.K = M.E / (1.0 - 2.0 * M.nu) / 3.0;
    M.lambda = 2.0 * M.G * M.nu / (1.0 - 2.0 * M.nu);
    M.wos = std::sqrt((M.lambda + 2.0 * M.G) / M.rho);
    M.yield0 = mat->yield_stress;
    M.hardening = mat->hardening_modulus;
    M.plastic = mat->yield_stress > 0.0 ? 1 : 0;
    M.c_dr = params->c_dr;
    M.c_cr = params->c_cr;
    M.cvisl = params->cvisl;
    M.cvisq = params->cvisq;
    M.gravity_on = params->gravity_on;
    M.gravity_value = params->gravity_value;
    for (int i = 0; i < 3; ++i) M.gravity_dir[i] = params->gravity_dir[i];
    // the amplitude table stays in the caller's device memory; the node pass
    // reads it there
    M.amp = m->gravity_amp_n > 0 ? m->gravity_amp : nullptr;
    M.amp_n = m->gravity_amp_n;
    ensc::set_mixed_consts(M);

    // the shared scratch keeps the previous call's contents: every control
    // field is rewritten here, reductions restart from +inf, sums from zero
    ensc::Ctl c{};
    c.time = clk->time;
    c.dt_i = clk->dt_i;
    c.dt_i_1 = clk->dt_i_1;
    c.step_end = step_end_time;
    c.pause_time = HUGE_VAL;
    c.total_time = params->total_time;
    c.factor = params->factor_timestep;
    c.wos = M.wos;
    c.len_min = ensc::kInfBits;
    if (clk->init_pass || !(clk->dt_stable_min > 0.0)) {
        c.dts_next = ensc::kInfBits;
    } else {
        std::memcpy(&c.dts_next, &clk->dt_stable_min, sizeof(double));
    }
    c.cycles_target = max_cycles;
    cudaError_t e = cudaMemcpyAsync(ctl, &c, sizeof(c), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(ENSC_ERR_CUDA, std::string("control upload: ") + cudaGetErrorString(e));

    const int ge = P.n_elem_blocks, gn = P.n_node_blocks;
    // the work partials accumulate over the call's cycles
    e = cudaMemsetAsync(P.elem, 0, kPartialBytes, st);
    if (e != cudaSuccess) return fail(ENSC_ERR_CUDA, std::string("partials reset: ") + cudaGetErrorString(e));
    // init()'s force pass sees the velocities before any boundary condition
    // (exDyna3D.cpp:124-141); the step's conditions are then applied to the
    // velocity field, as setCurrentStep / computeSate do (:1911, :782)
    if (clk->init_pass) ensc::launch_element_fp64(E, N, M, ctl, P, ge, true, st);
    ensc::launch_apply_bc_v(N, false, st);
    // cycles in batches; after each, the control block tells whether the run
    // stopped (step end reached, cycle budget spent, or a status raised)
    int64_t launched = 0;
    while (launched < max_cycles) {
        const int64_t n = std::min<int64_t>(kBatchCycles, max_cycles - launched);
        for (int64_t i = 0; i < n; ++i) {
            ensc::launch_between(ctl, P, 0, st);
            ensc::launch_edge_prepass(E, N, ctl, ge, st);
            ensc::launch_element_fp64(E, N, M, ctl, P, ge, false, st);
            ensc::launch_node_fp64(E, N, M, ctl, P, gn, st);
        }
        launched += n;
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(ENSC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
        e = cudaMemcpyAsync(&c, ctl, sizeof(c), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(ENSC_ERR_CUDA, std::string("control read-back: ") + cudaGetErrorString(e));
        if (c.status || !(c.time < c.step_end) || c.cycles_done >= max_cycles) break;
    }
    ensc::launch_between(ctl, P, 1, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ENSC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    e = cudaMemcpyAsync(&c, ctl, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(ENSC_ERR_CUDA, std::string("control read-back: ") + cudaGetErrorString(e));
    clk->time = c.time;
    clk->dt_i = c.dt_i;
    clk->dt_i_1 = c.dt_i_1;
    std::memcpy(&clk->dt_stable_min, &c.dts_next, sizeof(double));
    clk->init_pass = 0;
    clk->cycles = c.cycles_done;
    if (c.status & ensc::ST_NONFINITE) return fail(ENSC_ERR_NONFINITE, "non-finite nodal state detected");
    if (c.status & ensc::ST_INVERTED) return fail(ENSC_ERR_INVERTED, "element with J <= 0 detected");
    if (c.status & ensc::ST_BAD_DT) return fail(ENSC_ERR_NONFINITE, "stable time step is not positive");
    return ENSC_OK;
}

}  // extern "C"
