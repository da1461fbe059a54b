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
    ensc::Material M{};
    ensc::Partials P{};
    Ctl* ctl = nullptr;            // device
    Ctl* ctl_host = nullptr;       // pinned mirror
    int grid_e = 1, grid_n = 1;
    int chunk = 32;
    cudaGraphExec_t graph = nullptr;
    bool kinetic0_done = false;
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

int64_t pad32(int64_t n) { return (n + 31) / 32 * 32; }

// Restatement of compute_invMassMatrix (exDyna3D.cpp:492-515) with
// FEValues::reinit at the single Gauss point (fevalues.h:232-265): J = dN X,
// B = J^-1 dN, V0 = det(J) * 8, node mass += rho V0 / 8 in element order.
// The 3x3 determinant and inverse are Eigen 3.4's closed forms, the library
// the reference uses.
double det3h(const double m[3][3]) {
    const double h0 = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    const double h1 = m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    const double h2 = m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    return (h0 - h1) + h2;
}
double cof3h(const double m[3][3], int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
}
void inv3h(const double m[3][3], double r[3][3]) {
    const double c0 = cof3h(m, 0, 0), c1 = cof3h(m, 1, 0), c2 = cof3h(m, 2, 0);
    const double det = (c0 * m[0][0] + c1 * m[1][0]) + c2 * m[2][0];
    const double invdet = 1.0 / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = cof3h(m, j, i) * invdet;
}

void element_constants(int64_t nn, int64_t ne, const uint32_t* conn, const double* x0, double rho,
                       std::vector<double>& bt, std::vector<double>& vol0, std::vector<double>& inv_mass) {
    static const double XI[8][3] = {{-1., -1., -1.}, {1., -1., -1.}, {1., 1., -1.}, {-1., 1., -1.},
                                    {-1., -1., 1.},  {1., -1., 1.},  {1., 1., 1.},  {-1., 1., 1.}};
    double dn[3][8];
    for (int a = 0; a < 8; ++a)
        for (int d = 0; d < 3; ++d) dn[d][a] = 1.0 / 8.0 * XI[a][d];
    bt.assign(static_cast<size_t>(24 * ne), 0.0);
    vol0.assign(static_cast<size_t>(ne), 0.0);
    std::vector<double> mass(static_cast<size_t>(3 * nn), 0.0);
    for (int64_t e = 0; e < ne; ++e) {
        double xyz[8][3];
        for (int a = 0; a < 8; ++a)
            for (int c = 0; c < 3; ++c) xyz[a][c] = x0[3 * static_cast<int64_t>(conn[8 * e + a]) + c];
        double jac[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double s = dn[r][0] * xyz[0][c];
                for (int k = 1; k < 8; ++k) s += dn[r][k] * xyz[k][c];
                jac[r][c] = s;
            }
        double ij[3][3];
        inv3h(jac, ij);
        const double detj = det3h(jac);
        for (int a = 0; a < 8; ++a)
            for (int r = 0; r < 3; ++r)
                bt[24 * e + 3 * a + r] = (ij[r][0] * dn[0][a] + ij[r][1] * dn[1][a]) + ij[r][2] * dn[2][a];
        const double v0 = detj * 8.0;
        vol0[e] = v0;
        const double nm = rho * v0 / 8.0;
        for (int a = 0; a < 8; ++a)
            for (int c = 0; c < 3; ++c) mass[3 * static_cast<int64_t>(conn[8 * e + a]) + c] += nm;
    }
    inv_mass.resize(static_cast<size_t>(3 * nn));
    for (int64_t i = 0; i < 3 * nn; ++i) inv_mass[i] = 1.0 / mass[i];
}

template <typename T>
int upload(ensc_handle* h, void* dst, const std::vector<T>& src) {
    if (src.empty()) return ENSC_OK;
    CK(h, cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return ENSC_OK;
}

// Converts an AoS host array [n][comps] into SoA [comps][pad] of type T.
template <typename T>
std::vector<T> to_soa(const double* aos, int64_t n, int64_t pad, int comps) {
    std::vector<T> out(static_cast<size_t>(comps * pad), T(0));
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < comps; ++c) out[c * pad + i] = static_cast<T>(aos[i * comps + c]);
    return out;
}

bool mixed(const ensc_handle* h) { return h->precision == ENSC_MIXED; }

void launch_element(ensc_handle* h, bool init, cudaStream_t st) {
    if (mixed(h)) ensc::launch_element_mixed(h->E, h->N, h->M, h->ctl, h->P, h->grid_e, init, st);
    else ensc::launch_element_fp64(h->E, h->N, h->M, h->ctl, h->P, h->grid_e, init, st);
}

void launch_node(ensc_handle* h, cudaStream_t st) {
    if (mixed(h)) ensc::launch_node_mixed(h->E, h->N, h->M, h->ctl, h->P, h->grid_n, st);
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
        ensc::launch_begin_exact(h->ctl, h->cap_stream);
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
    r->status = c.status ? ((c.status & ensc::ST_INVERTED) ? ENSC_ERR_INVERTED : ENSC_ERR_NONFINITE) : 0;
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
    if (mesh->n_nodes <= 0 || mesh->n_elements <= 0 || !mesh->conn || !mesh->x0)
        return set_err(nullptr, ENSC_ERR_ARG, "empty mesh or missing conn/x0");
    if (mesh->n_nodes >= (int64_t(1) << 32) - 1 || mesh->n_elements >= (int64_t(1) << 29))
        return set_err(nullptr, ENSC_ERR_ARG, "mesh too large for 32-bit node / 29-bit element indices");
    if (params->precision != ENSC_FP64 && params->precision != ENSC_MIXED)
        return set_err(nullptr, ENSC_ERR_ARG, "unsupported precision");
    if (!(mat->rho > 0.0) || !(mat->E > 0.0) || !(mat->nu < 0.5))
        return set_err(nullptr, ENSC_ERR_ARG, "invalid material");
    if (!(params->factor_timestep > 0.0)) return set_err(nullptr, ENSC_ERR_ARG, "factor_timestep must be > 0");
    const int64_t nn = mesh->n_nodes, ne = mesh->n_elements;
    for (int64_t i = 0; i < 8 * ne; ++i)
        if (static_cast<int64_t>(mesh->conn[i]) >= nn)
            return set_err(nullptr, ENSC_ERR_ARG, "connectivity index out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= params->device || params->device < 0)
        return set_err(nullptr, ENSC_ERR_NODEVICE, "no usable CUDA device");

    ensc_handle* h = new ensc_handle();
    h->device = params->device;
    h->precision = params->precision;
    h->plastic = mat->yield_stress > 0.0;
    h->nn = nn;
    h->ne = ne;
    h->nn_pad = pad32(nn);
    h->ne_pad = pad32(ne);
    h->chunk = params->graph_chunk > 0 ? params->graph_chunk : 32;
    DevGuard dg(h->device);
    auto fail = [&](int code) {
        g_create_error = h->err;
        ensc_destroy(h);
        return code;
    };

    // ---- element constants and lumped mass (host) ----
    std::vector<double> bt, vol0, inv_mass_dof;
    if (mesh->bt && mesh->vol0 && mesh->inv_mass) {
        bt.assign(mesh->bt, mesh->bt + 24 * ne);
        vol0.assign(mesh->vol0, mesh->vol0 + ne);
        inv_mass_dof.assign(mesh->inv_mass, mesh->inv_mass + 3 * nn);
    } else {
        element_constants(nn, ne, mesh->conn, mesh->x0, mat->rho, bt, vol0, inv_mass_dof);
    }
    std::vector<double> cb(ne), cb2(ne), im(h->nn_pad, 1.0);
    for (int64_t e = 0; e < ne; ++e) {
        cb[e] = std::cbrt(vol0[e]);
        cb2[e] = std::cbrt(vol0[e] * vol0[e]);
    }
    for (int64_t n = 0; n < nn; ++n) im[n] = inv_mass_dof[3 * n];

    // ---- node-centric gather tables ----
    std::vector<uint32_t> ell(static_cast<size_t>(8 * h->nn_pad), ENSC_NONE);
    bool clash = false;
    for (int k = 0; k < 8 && !clash; ++k)
        for (int64_t e = 0; e < ne; ++e) {
            uint32_t& slot = ell[k * h->nn_pad + mesh->conn[8 * e + k]];
            if (slot != ENSC_NONE) {
                clash = true;
                break;
            }
            slot = static_cast<uint32_t>(e);
        }
    // per-node mask of occupied local slots (slot-major force hand-off)
    std::vector<uint8_t> slot_mask;
    if (!clash) {
        slot_mask.assign(static_cast<size_t>(h->nn_pad), 0);
        for (int k = 0; k < 8; ++k)
            for (int64_t n = 0; n < nn; ++n)
                if (ell[k * h->nn_pad + n] != ENSC_NONE) slot_mask[n] |= static_cast<uint8_t>(1u << k);
    }
    std::vector<int64_t> csr_ptr;
    std::vector<uint32_t> csr_ent;
    if (clash) {
        csr_ptr.assign(static_cast<size_t>(nn + 1), 0);
        for (int64_t i = 0; i < 8 * ne; ++i) csr_ptr[mesh->conn[i] + 1] += 1;
        for (int64_t n = 0; n < nn; ++n) csr_ptr[n + 1] += csr_ptr[n];
        csr_ent.resize(static_cast<size_t>(8 * ne));
        std::vector<int64_t> fill(csr_ptr.begin(), csr_ptr.end() - 1);
        for (int k = 0; k < 8; ++k)
            for (int64_t e = 0; e < ne; ++e) {
                const uint32_t n = mesh->conn[8 * e + k];
                csr_ent[fill[n]++] = (static_cast<uint32_t>(e) << 3) | static_cast<uint32_t>(k);
            }
    }

    // ---- launch geometry ----
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) {
        set_err(h, ENSC_ERR_CUDA, "cudaGetDeviceProperties failed");
        return fail(ENSC_ERR_CUDA);
    }
    const bool mx = h->precision == ENSC_MIXED;
    const int occ_e = std::max(1, mx ? ensc::occupancy_element_mixed(h->plastic) : ensc::occupancy_element_fp64(h->plastic));
    const int occ_n = std::max(1, mx ? ensc::occupancy_node_mixed() : ensc::occupancy_node_fp64());
    const int64_t ge = (ne + ensc::kElemThreads - 1) / ensc::kElemThreads;
    const int64_t gn = (nn + ensc::kNodeThreads - 1) / ensc::kNodeThreads;
    h->grid_e = static_cast<int>(std::min<int64_t>(ge, static_cast<int64_t>(occ_e) * prop.multiProcessorCount));
    h->grid_n = static_cast<int>(std::min<int64_t>(gn, static_cast<int64_t>(occ_n) * prop.multiProcessorCount));

    // ---- one device arena, every array 256-byte aligned ----
    const int64_t ep = h->ne_pad, np = h->nn_pad;
    const size_t real = mx ? 4 : 8;   // storage width of element state, forces and velocity
    struct Piece {
        void** dst;
        size_t bytes;
    };
    void *p_conn, *p_bt, *p_vol0, *p_cb, *p_cb2, *p_sig, *p_qia, *p_eps, *p_fe, *p_x, *p_u, *p_v, *p_im, *p_bc,
        *p_bcv, *p_ell, *p_rf, *p_pe, *p_pn, *p_ctl, *p_cptr = nullptr, *p_cent = nullptr, *p_mask = nullptr;
    const int64_t fe_rows = clash ? ep : np;   // slot-major hand-off is indexed by node
    std::vector<Piece> pieces = {
        {&p_conn, 8 * ep * sizeof(uint32_t)}, {&p_bt, 24 * ep * real}, {&p_vol0, ep * 8}, {&p_cb, ep * 8},
        {&p_cb2, ep * 8}, {&p_sig, 6 * ep * real}, {&p_qia, 12 * ep * real}, {&p_eps, ep * real},
        {&p_fe, static_cast<size_t>(24 * fe_rows) * real}, {&p_x, 3 * np * 8}, {&p_u, 3 * np * 8}, {&p_v, 3 * np * real},
        {&p_im, np * 8}, {&p_bc, static_cast<size_t>(np)}, {&p_bcv, 3 * np * 8},
        {&p_ell, 8 * np * sizeof(uint32_t)}, {&p_rf, 3 * np * 8},
        {&p_pe, 3 * static_cast<size_t>(h->grid_e) * 8}, {&p_pn, 2 * static_cast<size_t>(h->grid_n) * 8},
        {&p_ctl, sizeof(Ctl)}};
    if (clash) {
        pieces.push_back({&p_cptr, (nn + 1) * sizeof(int64_t)});
        pieces.push_back({&p_cent, 8 * ne * sizeof(uint32_t)});
    } else {
        pieces.push_back({&p_mask, static_cast<size_t>(np)});
    }
    size_t total = 0;
    for (auto& pc : pieces) total += (pc.bytes + 255) / 256 * 256;
    cudaError_t ce = cudaMalloc(&h->arena, total);
    if (ce != cudaSuccess) {
        cuda_err(h, "cudaMalloc(arena)", ce);
        return fail(ENSC_ERR_OOM);
    }
    h->arena_bytes = total;
    {
        char* base = static_cast<char*>(h->arena);
        size_t off = 0;
        for (auto& pc : pieces) {
            *pc.dst = base + off;
            off += (pc.bytes + 255) / 256 * 256;
        }
    }
    ce = cudaMemset(h->arena, 0, total);
    if (ce != cudaSuccess) {
        cuda_err(h, "cudaMemset(arena)", ce);
        return fail(ENSC_ERR_CUDA);
    }
    // staging for AoS up/download: reuse the element force scratch when large enough
    const size_t need_stage = std::max<size_t>(12 * ne, 3 * nn) * sizeof(double);
    if (static_cast<size_t>(24 * fe_rows) * real >= need_stage) {
        h->staging = static_cast<double*>(p_fe);
    } else {
        ce = cudaMalloc(reinterpret_cast<void**>(&h->staging), need_stage);
        if (ce != cudaSuccess) {
            cuda_err(h, "cudaMalloc(staging)", ce);
            return fail(ENSC_ERR_OOM);
        }
        h->staging_owned = true;
    }
    h->staging_bytes = need_stage;
    if (cudaMallocHost(reinterpret_cast<void**>(&h->ctl_host), sizeof(Ctl)) != cudaSuccess) {
        set_err(h, ENSC_ERR_OOM, "cudaMallocHost(ctl)");
        return fail(ENSC_ERR_OOM);
    }

    // ---- arrays ----
    h->E.ne = ne;
    h->E.ne_pad = ep;
    h->E.conn = static_cast<uint32_t*>(p_conn);
    h->E.bt = p_bt;
    h->E.vol0 = static_cast<double*>(p_vol0);
    h->E.cbrt_v0 = static_cast<double*>(p_cb);
    h->E.cbrt_v0sq = static_cast<double*>(p_cb2);
    h->E.sigma = p_sig;
    h->E.qia = p_qia;
    h->E.eps_p = p_eps;
    h->E.fe = p_fe;
    h->E.tiles_aligned = 1;  // arena pieces are 256-byte aligned, ne_pad % 32 == 0
    h->E.slot_major = clash ? 0 : 1;
    h->N.nn = nn;
    h->N.nn_pad = np;
    h->N.x = static_cast<double*>(p_x);
    h->N.u = static_cast<double*>(p_u);
    h->N.v = p_v;
    h->N.inv_mass = static_cast<double*>(p_im);
    h->N.bc = static_cast<uint8_t*>(p_bc);
    h->N.bcv = static_cast<double*>(p_bcv);
    h->N.ell = static_cast<uint32_t*>(p_ell);
    h->N.csr_ptr = clash ? static_cast<int64_t*>(p_cptr) : nullptr;
    h->N.csr_ent = clash ? static_cast<uint32_t*>(p_cent) : nullptr;
    h->N.rf = static_cast<double*>(p_rf);
    h->N.slot_mask = clash ? nullptr : static_cast<uint8_t*>(p_mask);
    h->P.elem = static_cast<double*>(p_pe);
    h->P.node = static_cast<double*>(p_pn);
    h->P.n_elem_blocks = h->grid_e;
    h->P.n_node_blocks = h->grid_n;
    h->ctl = static_cast<Ctl*>(p_ctl);

    {
        std::vector<uint32_t> conn_soa(static_cast<size_t>(8 * ep), 0);
        for (int64_t e = 0; e < ne; ++e)
            for (int k = 0; k < 8; ++k) conn_soa[k * ep + e] = mesh->conn[8 * e + k];
        int rc = upload(h, p_conn, conn_soa);
        if (rc) return fail(rc);
        if (mx) {
            rc = upload(h, p_bt, to_soa<float>(bt.data(), ne, ep, 24));
            std::vector<float> v0f(vol0.begin(), vol0.end()), cbf(cb.begin(), cb.end());
            if (!rc) rc = upload(h, p_vol0, v0f);
            if (!rc) rc = upload(h, p_cb, cbf);
        } else {
            rc = upload(h, p_bt, to_soa<double>(bt.data(), ne, ep, 24));
            if (!rc) rc = upload(h, p_vol0, vol0);
            if (!rc) rc = upload(h, p_cb, cb);
            if (!rc) rc = upload(h, p_cb2, cb2);
        }
        if (rc) return fail(rc);
        if (!rc) rc = upload(h, p_im, im);
        if (!rc) rc = upload(h, p_x, to_soa<double>(mesh->x0, nn, np, 3));
        if (!rc && mesh->v0) {
            rc = mx ? upload(h, p_v, to_soa<float>(mesh->v0, nn, np, 3))
                    : upload(h, p_v, to_soa<double>(mesh->v0, nn, np, 3));
        }
        if (!rc) rc = upload(h, p_ell, ell);
        if (!rc && clash) rc = upload(h, p_cptr, csr_ptr);
        if (!rc && clash) rc = upload(h, p_cent, csr_ent);
        if (!rc && !clash) rc = upload(h, p_mask, slot_mask);
        if (rc) return fail(rc);
    }

    // ---- material and controls (Material_elastic::update, Material_elastic.cpp:9-14) ----
    ensc::Material& M = h->M;
    M.E = mat->E;
    M.nu = mat->nu;
    M.rho = mat->rho;
    M.G = M.E / ((1.0 + M.nu) * 2.0);
    M.K = M.E / (1.0 - 2.0 * M.nu) / 3.0;
    M.lambda = 2.0 * M.G * M.nu / (1.0 - 2.0 * M.nu);
    M.wos = std::sqrt((M.lambda + 2.0 * M.G) / M.rho);
    M.yield0 = mat->yield_stress;
    M.hardening = mat->hardening_modulus;
    M.plastic = h->plastic ? 1 : 0;
    M.c_dr = params->c_dr;
    M.c_cr = params->c_cr;
    M.cvisl = params->cvisl;
    M.cvisq = params->cvisq;
    M.gravity_on = params->gravity_on;
    M.gravity_value = params->gravity_value;
    for (int i = 0; i < 3; ++i) M.gravity_dir[i] = params->gravity_dir[i];

    Ctl c{};
    c.time = 0.0;
    c.dt_i = 0.0;
    c.dt_i_1 = 0.0;
    c.step_end = HUGE_VAL;
    c.total_time = params->total_time;
    c.factor = params->factor_timestep;
    c.wos = M.wos;
    c.dts_next = ensc::kInfBits;
    c.len_min = ensc::kInfBits;
    *h->ctl_host = c;

    // ---- streams ----
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
    int rc = build_graph(h);
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

int ensc_step_async(ensc_handle* h, int64_t max_cycles, double step_end_time) {
    if (!h || max_cycles < 0) return ENSC_ERR_ARG;
    if (max_cycles == 0) return ENSC_OK;
    DevGuard dg(h->device);
    ensc::launch_arm(h->ctl, step_end_time, max_cycles, h->stream);
    const int64_t launches = (max_cycles + h->chunk - 1) / h->chunk;
    for (int64_t i = 0; i < launches; ++i) CK(h, cudaGraphLaunch(h->graph, h->stream));
    CK(h, cudaGetLastError());
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
    if (!h || max_cycles < 0) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    const int64_t before = h->ctl_host->cycles_done;
    if (max_cycles > 0) {
        ensc::launch_arm(h->ctl, step_end_time, max_cycles, h->stream);
        // launch graphs in batches; between batches read the control block
        // to stop once time reached step_end
        const int64_t batch = std::max<int64_t>(1, 4096 / h->chunk);
        int64_t launched = 0;
        const int64_t needed = (max_cycles + h->chunk - 1) / h->chunk;
        while (launched < needed) {
            const int64_t n = std::min(batch, needed - launched);
            for (int64_t i = 0; i < n; ++i) CK(h, cudaGraphLaunch(h->graph, h->stream));
            launched += n;
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

int ensc_download(ensc_handle* h, double* x, double* u, double* v, double* sigma, double* qia, double* eps_p) {
    if (!h) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    struct Item {
        double* dst;
        const void* src;
        int64_t n, pad;
        int comps;
        bool f32;
    };
    const bool mx = mixed(h);
    const Item items[] = {{x, h->N.x, h->nn, h->nn_pad, 3, false},        {u, h->N.u, h->nn, h->nn_pad, 3, false},
                          {v, h->N.v, h->nn, h->nn_pad, 3, mx},           {sigma, h->E.sigma, h->ne, h->ne_pad, 6, mx},
                          {qia, h->E.qia, h->ne, h->ne_pad, 12, mx},      {eps_p, h->E.eps_p, h->ne, h->ne_pad, 1, mx}};
    for (const Item& it : items) {
        if (!it.dst) continue;
        ensc::launch_soa_to_aos(it.src, it.n, it.pad, it.comps, it.f32, h->staging, h->stream);
        CK(h, cudaGetLastError());
        CK(h, cudaMemcpyAsync(it.dst, h->staging, it.n * it.comps * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    return ENSC_OK;
}

int ensc_download_reactions(ensc_handle* h, double* rf) {
    if (!h || !rf) return ENSC_ERR_ARG;
    DevGuard dg(h->device);
    ensc::launch_soa_to_aos(h->N.rf, h->nn, h->nn_pad, 3, false, h->staging, h->stream);
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(rf, h->staging, h->nn * 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return ENSC_OK;
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
    };
    const bool mx = mixed(h);
    const Item items[] = {{x, h->N.x, h->nn, h->nn_pad, 3, false},        {u, h->N.u, h->nn, h->nn_pad, 3, false},
                          {v, h->N.v, h->nn, h->nn_pad, 3, mx},           {sigma, h->E.sigma, h->ne, h->ne_pad, 6, mx},
                          {qia, h->E.qia, h->ne, h->ne_pad, 12, mx},      {eps_p, h->E.eps_p, h->ne, h->ne_pad, 1, mx}};
    for (const Item& it : items) {
        if (!it.src) continue;
        CK(h, cudaMemcpyAsync(h->staging, it.src, it.n * it.comps * sizeof(double), cudaMemcpyHostToDevice,
                              h->stream));
        ensc::launch_aos_to_soa(h->staging, it.n, it.pad, it.comps, it.dst, it.f32, h->stream);
        CK(h, cudaGetLastError());
    }
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
        ensc::launch_begin_exact(h->ctl, h->stream);
        cudaEventRecord(ev[3], h->stream);
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

int32_t ensc_kernels_per_cycle(const ensc_handle* h) { return h ? 5 : 0; }

void ensc_destroy(ensc_handle* h) {
    if (!h) return;
    DevGuard dg(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    if (h->staging_owned && h->staging) cudaFree(h->staging);
    if (h->arena) cudaFree(h->arena);
    if (h->ctl_host) cudaFreeHost(h->ctl_host);
    delete h;
}

}  // extern "C"
