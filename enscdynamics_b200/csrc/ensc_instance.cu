// Host-side preparation and device layout of one solver instance.
#include "ensc_instance.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace ensc {
namespace {

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

// Converts an AoS host array [n][comps] into SoA [comps][pad] of type T.
template <typename T>
std::vector<T> to_soa(const double* aos, int64_t n, int64_t pad, int comps) {
    std::vector<T> out(static_cast<size_t>(comps * pad), T(0));
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < comps; ++c) out[c * pad + i] = static_cast<T>(aos[i * comps + c]);
    return out;
}

// The rows the upload copies as they are (InstanceHost::a_rows ...): the
// element geometry in the precision's device form, x0 and v0 as SoA rows.
// The caller's x0 and v0 are not read after this.
void form_device_rows(InstanceHost& h) {
    const int64_t ep = h.ne_pad, np = h.nn_pad;
    if (h.mixed) {
        // corner signs s_j of the reference hexahedron (Element_HexN8.cpp:49-91)
        static const double kCorner[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                             {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
        h.a_rows.assign(static_cast<size_t>(18 * ep), 0.f);
        for (int64_t el = 0; el < h.ne; ++el)
            for (int c = 0; c < 3; ++c)
                for (int m = 0; m < 3; ++m) {
                    double v = 0.0;
                    for (int j = 0; j < 8; ++j) v += h.bt[24 * el + 3 * j + c] * kCorner[j][m];
                    const float hi = static_cast<float>(v);
                    h.a_rows[(3 * c + m) * ep + el] = hi;
                    h.a_rows[(9 + 3 * c + m) * ep + el] = static_cast<float>(v - static_cast<double>(hi));
                }
        h.cb_f.assign(h.cb.begin(), h.cb.end());
    } else {
        h.bt_rows = to_soa<double>(h.bt.data(), h.ne, ep, 24);
    }
    std::vector<double>().swap(h.bt);  // the device form replaces it
    h.x_rows = to_soa<double>(h.x0, h.nn, np, 3);
    if (h.v0) {
        if (h.mixed) {
            h.v_rows_f = to_soa<float>(h.v0, h.nn, np, 3);
#if ENSC_MIXED_VLO
            h.v_lo_rows.assign(static_cast<size_t>(3 * np), 0);
            for (int64_t n = 0; n < h.nn; ++n)
                for (int c = 0; c < 3; ++c) v_split(h.v0[3 * n + c], h.v_rows_f[c * np + n], h.v_lo_rows[c * np + n]);
#endif
        } else {
            h.v_rows_d = to_soa<double>(h.v0, h.nn, np, 3);
        }
    }
    h.x0 = nullptr;
    h.v0 = nullptr;
}

template <typename T>
cudaError_t put(void* block, size_t off, const std::vector<T>& v, cudaStream_t st) {
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(static_cast<char*>(block) + off, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                           st);
}

}  // namespace

std::vector<int32_t> patch_order(int64_t ne, const uint32_t* conn, const double* x0) {
    std::vector<double> cen(static_cast<size_t>(3 * ne));
    double lo[3], hi[3], ext[3];
    for (int c = 0; c < 3; ++c) {
        lo[c] = std::numeric_limits<double>::infinity();
        hi[c] = -lo[c];
        ext[c] = lo[c];
    }
    for (int64_t e = 0; e < ne; ++e)
        for (int c = 0; c < 3; ++c) {
            double sum = 0.0, mn = std::numeric_limits<double>::infinity(), mx = -mn;
            for (int k = 0; k < 8; ++k) {
                const double v = x0[3 * static_cast<int64_t>(conn[8 * e + k]) + c];
                sum += v;
                mn = std::min(mn, v);
                mx = std::max(mx, v);
            }
            const double m = sum / 8.0;
            cen[3 * e + c] = m;
            lo[c] = std::min(lo[c], m);
            hi[c] = std::max(hi[c], m);
            if (mx - mn > 0.0) ext[c] = std::min(ext[c], mx - mn);
        }
    // cell size per axis: the smallest element extent, widened so that the
    // cell indices fit 21 bits; centroids of a structured grid land on whole
    // cells
    constexpr double kMaxCell = (1 << 21) - 1;
    double hc[3];
    for (int c = 0; c < 3; ++c) {
        const double range = hi[c] - lo[c];
        hc[c] = std::isfinite(ext[c]) ? ext[c] : 1.0;
        if (range / hc[c] > kMaxCell) hc[c] = range / kMaxCell;
    }
    std::vector<std::pair<uint64_t, int32_t>> key(static_cast<size_t>(ne));
    for (int64_t e = 0; e < ne; ++e) {
        uint64_t cell[3];
        for (int c = 0; c < 3; ++c) {
            const double t = std::floor((cen[3 * e + c] - lo[c]) / hc[c] + 0.5);
            cell[c] = static_cast<uint64_t>(std::min(std::max(t, 0.0), kMaxCell));
        }
        uint64_t m = 0;
        for (int b = 0; b < 21; ++b)
            for (int c = 0; c < 3; ++c) m |= ((cell[c] >> b) & 1u) << (3 * b + c);
        key[e] = {m, static_cast<int32_t>(e)};
    }
    std::sort(key.begin(), key.end());
    std::vector<int32_t> perm(static_cast<size_t>(ne));
    for (int64_t s = 0; s < ne; ++s) perm[s] = key[s].second;
    return perm;
}

void build_patches(int64_t nn, int64_t ne, const uint32_t* conn, InstanceHost& h) {
    const int64_t npatch = (ne + kPatchElems - 1) / kPatchElems;
    h.n_patches = npatch;
    h.pf_off.assign(static_cast<size_t>(npatch + 1), 0);
    h.pinc.assign(static_cast<size_t>(8 * ne), 0);
    h.pinc_off.clear();
    h.pinc_off.reserve(static_cast<size_t>(2 * nn + npatch + 1));
    std::vector<uint32_t> pnode;
    pnode.reserve(static_cast<size_t>(2 * nn + npatch));
    std::vector<uint64_t> trip;
    trip.reserve(8 * kPatchElems);
    uint32_t pos = 0;
    for (int64_t p = 0; p < npatch; ++p) {
        const int64_t e0 = p * kPatchElems, e1 = std::min(ne, e0 + kPatchElems);
        trip.clear();
        // (node, slot, element in patch), sorted: each node's incidences in
        // slot order
        for (int64_t e = e0; e < e1; ++e)
            for (int k = 0; k < 8; ++k)
                trip.push_back((static_cast<uint64_t>(conn[8 * e + k]) << 32) | (static_cast<uint64_t>(k) << 8) |
                               static_cast<uint64_t>(e - e0));
        std::sort(trip.begin(), trip.end());
        h.pf_off[p] = static_cast<uint32_t>(pnode.size());
        for (size_t i = 0; i < trip.size(); ++i) {
            const uint32_t node = static_cast<uint32_t>(trip[i] >> 32);
            if (i == 0 || node != static_cast<uint32_t>(trip[i - 1] >> 32)) {
                pnode.push_back(node);
                h.pinc_off.push_back(pos);
            }
            const uint32_t k = static_cast<uint32_t>((trip[i] >> 8) & 7u), el = static_cast<uint32_t>(trip[i] & 0xffu);
            h.pinc[pos++] = static_cast<uint16_t>((el << 3) | k);
        }
    }
    h.pf_off[npatch] = static_cast<uint32_t>(pnode.size());
    h.pinc_off.push_back(pos);
    h.n_pnodes = static_cast<int64_t>(pnode.size());
    // node -> its partials, in patch order
    h.nptr.assign(static_cast<size_t>(nn + 1), 0);
    for (uint32_t g : pnode) h.nptr[g + 1] += 1;
    for (int64_t n = 0; n < nn; ++n) h.nptr[n + 1] += h.nptr[n];
    h.nent.resize(pnode.size());
    std::vector<uint32_t> fill(h.nptr.begin(), h.nptr.end() - 1);
    for (size_t q = 0; q < pnode.size(); ++q) h.nent[fill[pnode[q]]++] = static_cast<uint32_t>(q);
}

int instance_prepare(const ensc_mesh_desc* mesh, const ensc_material* mat, bool mixed, int assembly,
                     InstanceHost& h, std::string& err) {
    if (!mesh || !mat) {
        err = "mesh and material are required";
        return ENSC_ERR_ARG;
    }
    if (mesh->n_nodes <= 0 || mesh->n_elements <= 0 || !mesh->conn || !mesh->x0) {
        err = "empty mesh or missing conn/x0";
        return ENSC_ERR_ARG;
    }
    if (mesh->n_nodes >= (int64_t(1) << 32) - 1 || mesh->n_elements >= (int64_t(1) << 29)) {
        err = "mesh too large for 32-bit node / 29-bit element indices";
        return ENSC_ERR_ARG;
    }
    if (!(mat->rho > 0.0) || !(mat->E > 0.0) || !(mat->nu < 0.5)) {
        err = "invalid material";
        return ENSC_ERR_ARG;
    }
    const int64_t nn = mesh->n_nodes, ne = mesh->n_elements;
    for (int64_t i = 0; i < 8 * ne; ++i)
        if (static_cast<int64_t>(mesh->conn[i]) >= nn) {
            err = "connectivity index out of range";
            return ENSC_ERR_ARG;
        }
    h.nn = nn;
    h.ne = ne;
    h.nn_pad = pad32(nn);
    h.ne_pad = pad32(ne);
    h.mixed = mixed;
    h.plastic = mat->yield_stress > 0.0;
    h.x0 = mesh->x0;
    h.v0 = mesh->v0;
    const int64_t ep = h.ne_pad, np = h.nn_pad;

    // element constants and lumped mass, in the caller's element order (the
    // mass sums follow it)
    std::vector<double> inv_mass_dof;
    if (mesh->bt && mesh->vol0 && mesh->inv_mass) {
        h.bt.assign(mesh->bt, mesh->bt + 24 * ne);
        h.vol0.assign(mesh->vol0, mesh->vol0 + ne);
        inv_mass_dof.assign(mesh->inv_mass, mesh->inv_mass + 3 * nn);
    } else {
        element_constants(nn, ne, mesh->conn, mesh->x0, mat->rho, h.bt, h.vol0, inv_mass_dof);
    }

    // no node repeating a local slot: slot-major forces, and patches allowed
    h.clash = false;
    {
        std::vector<uint8_t> seen(static_cast<size_t>(nn), 0);
        for (int64_t e = 0; e < ne && !h.clash; ++e)
            for (int k = 0; k < 8; ++k) {
                uint8_t& m = seen[mesh->conn[8 * e + k]];
                if ((m >> k) & 1u) {
                    h.clash = true;
                    break;
                }
                m = static_cast<uint8_t>(m | (1u << k));
            }
    }
    if (assembly != ENSC_ASSEMBLY_AUTO && assembly != ENSC_ASSEMBLY_SLOT && assembly != ENSC_ASSEMBLY_PATCH) {
        err = "unknown force assembly";
        return ENSC_ERR_ARG;
    }
    if (assembly == ENSC_ASSEMBLY_PATCH && (!mixed || h.clash)) {
        err = "patch assembly needs mixed precision and a mesh where no node repeats a local slot";
        return ENSC_ERR_ARG;
    }
    h.patch = assembly == ENSC_ASSEMBLY_PATCH;

    // stored element order: the caller's, or patch order
    const uint32_t* conn = mesh->conn;
    std::vector<uint32_t> pconn;
    if (h.patch) {
        const std::vector<int32_t> perm = patch_order(ne, mesh->conn, mesh->x0);
        pconn.resize(static_cast<size_t>(8 * ne));
        std::vector<double> bt(static_cast<size_t>(24 * ne)), vol0(static_cast<size_t>(ne));
        h.iperm.resize(static_cast<size_t>(ne));
        for (int64_t sidx = 0; sidx < ne; ++sidx) {
            const int64_t e = perm[sidx];
            h.iperm[e] = static_cast<int32_t>(sidx);
            std::memcpy(&pconn[8 * sidx], &mesh->conn[8 * e], 8 * sizeof(uint32_t));
            std::memcpy(&bt[24 * sidx], &h.bt[24 * e], 24 * sizeof(double));
            vol0[sidx] = h.vol0[e];
        }
        h.bt.swap(bt);
        h.vol0.swap(vol0);
        conn = pconn.data();
        build_patches(nn, ne, conn, h);
    }

    h.cb.resize(ne);
    h.cb2.resize(ne);
    for (int64_t e = 0; e < ne; ++e) {
        h.cb[e] = std::cbrt(h.vol0[e]);
        h.cb2[e] = std::cbrt(h.vol0[e] * h.vol0[e]);
    }
    h.im.assign(static_cast<size_t>(np), 1.0);
    for (int64_t n = 0; n < nn; ++n) h.im[n] = inv_mass_dof[3 * n];
    h.conn_soa.assign(static_cast<size_t>(8 * ep), 0);
    for (int64_t e = 0; e < ne; ++e)
        for (int k = 0; k < 8; ++k) h.conn_soa[k * ep + e] = conn[8 * e + k];

    // node-to-element tables
    h.ell.assign(static_cast<size_t>(8 * np), ENSC_NONE);
    if (!h.clash) {
        for (int k = 0; k < 8; ++k)
            for (int64_t e = 0; e < ne; ++e) h.ell[k * np + conn[8 * e + k]] = static_cast<uint32_t>(e);
        h.slot_mask.assign(static_cast<size_t>(np), 0);
        for (int k = 0; k < 8; ++k)
            for (int64_t n = 0; n < nn; ++n)
                if (h.ell[k * np + n] != ENSC_NONE) h.slot_mask[n] |= static_cast<uint8_t>(1u << k);
    } else {
        // ell keeps the first element per (slot, node) as before; the lists
        // carry all of them
        for (int k = 0; k < 8; ++k)
            for (int64_t e = 0; e < ne; ++e) {
                uint32_t& slot = h.ell[k * np + conn[8 * e + k]];
                if (slot == ENSC_NONE) slot = static_cast<uint32_t>(e);
            }
        h.csr_ptr.assign(static_cast<size_t>(nn + 1), 0);
        for (int64_t i = 0; i < 8 * ne; ++i) h.csr_ptr[conn[i] + 1] += 1;
        for (int64_t n = 0; n < nn; ++n) h.csr_ptr[n + 1] += h.csr_ptr[n];
        h.csr_ent.resize(static_cast<size_t>(8 * ne));
        std::vector<int64_t> fill(h.csr_ptr.begin(), h.csr_ptr.end() - 1);
        for (int k = 0; k < 8; ++k)
            for (int64_t e = 0; e < ne; ++e) {
                const uint32_t n = conn[8 * e + k];
                h.csr_ent[fill[n]++] = (static_cast<uint32_t>(e) << 3) | static_cast<uint32_t>(k);
            }
    }

    // device layout
    const size_t real = mixed ? 4 : 8;  // element state, forces and velocity
    const size_t E8 = static_cast<size_t>(ep), N8 = static_cast<size_t>(np);
    const size_t fe_rows = h.clash ? E8 : N8;
    using P = InstanceHost::Piece;
    h.size[P::CONN] = 8 * E8 * sizeof(uint32_t);
    // FP64: B0^T rows as given; mixed: the 3x3 matrix A = sum_j B0_j s_j^T
    // (B0_j = A s_j / 8) as 9 hi and 9 lo float rows
    h.size[P::BT] = (mixed ? 18 : 24) * E8 * real;
    h.size[P::VOL0] = E8 * 8;
    h.size[P::CB] = E8 * 8;
    h.size[P::CB2] = E8 * 8;
    h.size[P::SIG] = 6 * E8 * real;
    h.size[P::QIA] = 12 * E8 * real;
    h.size[P::EPS] = E8 * real;
    h.size[P::FE] = 24 * fe_rows * real;
    h.size[P::X] = 3 * N8 * 8;
    h.size[P::U] = 3 * N8 * 8;
    // mixed: float rows, then the 16-bit velocity residual rows (v_lo_rows)
    h.size[P::V] = 3 * N8 * real + ((mixed && ENSC_MIXED_VLO) ? 3 * N8 * sizeof(int16_t) : 0);
    h.size[P::IM] = N8 * 8;
    h.size[P::BC] = N8;
    h.size[P::BCV] = 3 * N8 * 8;
    h.size[P::ELL] = 8 * N8 * sizeof(uint32_t);
    h.size[P::RF] = 3 * N8 * 8;
    h.size[P::CPTR] = h.clash ? static_cast<size_t>(nn + 1) * sizeof(int64_t) : 0;
    h.size[P::CENT] = h.clash ? static_cast<size_t>(8 * ne) * sizeof(uint32_t) : 0;
    h.size[P::MASK] = h.clash ? 0 : N8;
    if (h.patch) {
        h.size[P::IPERM] = static_cast<size_t>(ne) * sizeof(int32_t);
        h.size[P::PFOFF] = static_cast<size_t>(h.n_patches + 1) * sizeof(uint32_t);
        h.size[P::PINCOFF] = static_cast<size_t>(h.n_pnodes + 1) * sizeof(uint32_t);
        h.size[P::PINC] = static_cast<size_t>(8 * ne) * sizeof(uint16_t);
        h.size[P::PF] = 3 * static_cast<size_t>(pad32(h.n_pnodes)) * sizeof(float);
        // node groups read nptr[n0 .. n0 + W] with n0 + W <= nn_pad
        h.size[P::NPTR] = (N8 + 1) * sizeof(uint32_t);
        h.size[P::NENT] = static_cast<size_t>(h.n_pnodes) * sizeof(uint32_t);
    }
    size_t total = 0;
    for (int i = 0; i < P::NPIECE; ++i) {
        h.off[i] = total;
        total += (h.size[i] + 255) / 256 * 256;
    }
    h.bytes = total;
    form_device_rows(h);
    return ENSC_OK;
}

int instance_upload(const InstanceHost& h, void* block, cudaStream_t st, ElemArrays& E, NodeArrays& N,
                    PatchArrays& PA, std::string& err) {
    using P = InstanceHost::Piece;
    const int64_t ep = h.ne_pad, np = h.nn_pad;
    char* b = static_cast<char*>(block);
    cudaError_t e = cudaMemsetAsync(block, 0, h.bytes, st);
    if (h.mixed) {
        if (e == cudaSuccess) e = put(block, h.off[P::BT], h.a_rows, st);
        if (e == cudaSuccess) e = put(block, h.off[P::VOL0], h.vol0, st);
        if (e == cudaSuccess) e = put(block, h.off[P::CB], h.cb_f, st);
    } else {
        if (e == cudaSuccess) e = put(block, h.off[P::BT], h.bt_rows, st);
        if (e == cudaSuccess) e = put(block, h.off[P::VOL0], h.vol0, st);
        if (e == cudaSuccess) e = put(block, h.off[P::CB], h.cb, st);
        if (e == cudaSuccess) e = put(block, h.off[P::CB2], h.cb2, st);
    }
    if (e == cudaSuccess) e = put(block, h.off[P::CONN], h.conn_soa, st);
    if (e == cudaSuccess) e = put(block, h.off[P::IM], h.im, st);
    if (e == cudaSuccess) e = put(block, h.off[P::X], h.x_rows, st);
    // mixed: the u rows hold the reference position x - u, x0 at the start
    if (h.mixed && ENSC_MIXED_UREF && e == cudaSuccess) e = put(block, h.off[P::U], h.x_rows, st);
    if (h.mixed) {
        if (e == cudaSuccess) e = put(block, h.off[P::V], h.v_rows_f, st);
#if ENSC_MIXED_VLO
        if (e == cudaSuccess) e = put(block, h.off[P::V] + 3 * np * sizeof(float), h.v_lo_rows, st);
#endif
    } else {
        if (e == cudaSuccess) e = put(block, h.off[P::V], h.v_rows_d, st);
    }
    if (e == cudaSuccess) e = put(block, h.off[P::ELL], h.ell, st);
    if (h.clash) {
        if (e == cudaSuccess) e = put(block, h.off[P::CPTR], h.csr_ptr, st);
        if (e == cudaSuccess) e = put(block, h.off[P::CENT], h.csr_ent, st);
    } else {
        if (e == cudaSuccess) e = put(block, h.off[P::MASK], h.slot_mask, st);
    }
    std::vector<uint32_t> nptr_pad;
    if (h.patch) {
        // padding nodes have no partials: nptr stays at the total past nn
        nptr_pad.assign(static_cast<size_t>(np + 1), h.nptr.empty() ? 0u : h.nptr.back());
        std::copy(h.nptr.begin(), h.nptr.end(), nptr_pad.begin());
        if (e == cudaSuccess) e = put(block, h.off[P::IPERM], h.iperm, st);
        if (e == cudaSuccess) e = put(block, h.off[P::PFOFF], h.pf_off, st);
        if (e == cudaSuccess) e = put(block, h.off[P::PINCOFF], h.pinc_off, st);
        if (e == cudaSuccess) e = put(block, h.off[P::PINC], h.pinc, st);
        if (e == cudaSuccess) e = put(block, h.off[P::NPTR], nptr_pad, st);
        if (e == cudaSuccess) e = put(block, h.off[P::NENT], h.nent, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = std::string("instance upload: ") + cudaGetErrorString(e);
        return ENSC_ERR_CUDA;
    }
    E = ElemArrays{};
    E.ne = h.ne;
    E.ne_pad = ep;
    E.conn = reinterpret_cast<uint32_t*>(b + h.off[P::CONN]);
    E.bt = b + h.off[P::BT];
    E.vol0 = reinterpret_cast<double*>(b + h.off[P::VOL0]);
    E.cbrt_v0 = reinterpret_cast<double*>(b + h.off[P::CB]);
    E.cbrt_v0sq = reinterpret_cast<double*>(b + h.off[P::CB2]);
    E.sigma = b + h.off[P::SIG];
    E.qia = b + h.off[P::QIA];
    E.eps_p = b + h.off[P::EPS];
    E.fe = b + h.off[P::FE];
    E.tiles_aligned = 1;  // pieces are 256-byte aligned, ne_pad % 32 == 0
    E.slot_major = h.clash ? 0 : 1;
    PA = PatchArrays{};
    if (h.patch) {
        PA.pf_off = reinterpret_cast<uint32_t*>(b + h.off[P::PFOFF]);
        PA.pinc_off = reinterpret_cast<uint32_t*>(b + h.off[P::PINCOFF]);
        PA.pinc = reinterpret_cast<uint16_t*>(b + h.off[P::PINC]);
        PA.pf = reinterpret_cast<float*>(b + h.off[P::PF]);
        PA.pf_pad = pad32(h.n_pnodes);
        PA.nptr = reinterpret_cast<uint32_t*>(b + h.off[P::NPTR]);
        PA.nent = reinterpret_cast<uint32_t*>(b + h.off[P::NENT]);
        PA.iperm = reinterpret_cast<int32_t*>(b + h.off[P::IPERM]);
    }
    N = NodeArrays{};
    N.nn = h.nn;
    N.nn_pad = np;
    N.x = reinterpret_cast<double*>(b + h.off[P::X]);
    N.u = reinterpret_cast<double*>(b + h.off[P::U]);
    N.v = b + h.off[P::V];
    N.inv_mass = reinterpret_cast<double*>(b + h.off[P::IM]);
    N.bc = reinterpret_cast<uint8_t*>(b + h.off[P::BC]);
    N.bcv = reinterpret_cast<double*>(b + h.off[P::BCV]);
    N.ell = reinterpret_cast<uint32_t*>(b + h.off[P::ELL]);
    N.csr_ptr = h.clash ? reinterpret_cast<int64_t*>(b + h.off[P::CPTR]) : nullptr;
    N.csr_ent = h.clash ? reinterpret_cast<uint32_t*>(b + h.off[P::CENT]) : nullptr;
    N.rf = reinterpret_cast<double*>(b + h.off[P::RF]);
    N.slot_mask = h.clash ? nullptr : reinterpret_cast<uint8_t*>(b + h.off[P::MASK]);
    return ENSC_OK;
}

void material_from(const ensc_material* mat, const ensc_params* p, Material& M) {
    M = Material{};
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
    M.c_dr = p->c_dr;
    M.c_cr = p->c_cr;
    M.cvisl = p->cvisl;
    M.cvisq = p->cvisq;
    M.gravity_on = p->gravity_on;
    M.gravity_value = p->gravity_value;
    for (int i = 0; i < 3; ++i) M.gravity_dir[i] = p->gravity_dir[i];
    set_mixed_consts(M);
}

Ctl initial_ctl(const ensc_params* p, const Material& M) {
    Ctl c{};
    c.time = 0.0;
    c.dt_i = 0.0;
    c.dt_i_1 = 0.0;
    c.step_end = HUGE_VAL;
    c.pause_time = HUGE_VAL;
    c.total_time = p->total_time;
    c.factor = p->factor_timestep;
    c.wos = M.wos;
    c.dts_next = kInfBits;
    c.len_min = kInfBits;
    return c;
}

}  // namespace ensc
