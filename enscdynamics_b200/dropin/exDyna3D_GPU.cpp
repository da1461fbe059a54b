// exDyna3D_GPU: see exDyna3D_GPU.h.
#include "exDyna3D_GPU.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>

namespace EnSC {

namespace {

// Upper bound on the cycles one ensc_step_until call may run; the call
// returns earlier at the step end, the pause time or an error.
constexpr int64_t kCycleBound = int64_t(1) << 40;
// Most cycles enqueued ahead of an output write (ensc_step_until_async's
// limit is 2^24); the rest of the way runs after the write.
constexpr int64_t kAheadCycles = int64_t(1) << 20;

}  // namespace

exDyna3D_GPU::exDyna3D_GPU() : exDyna3D_GPU(Options()) {}

exDyna3D_GPU::exDyna3D_GPU(const Options& options) : opt_(options) {}

exDyna3D_GPU::~exDyna3D_GPU() {
    if (h_) ensc_destroy(h_);
}

void exDyna3D_GPU::check(int rc, const char* what) const {
    if (rc == ENSC_OK) return;
    throw std::runtime_error(std::string(what) + " failed (" + std::to_string(rc) + "): " +
                             ensc_last_error(h_));
}

// Hands the model as init() left it -- node coordinates, connectivity in the
// reference's local order, initial velocities, and the reference's own B0^T,
// V0 and inverse lumped mass (compute_invMassMatrix, exDyna3D.cpp:492-515) --
// to the device, with the controls read by read_project_txt (:698-772).
void exDyna3D_GPU::create_device() {
    const int64_t nn = static_cast<int64_t>(vertices.size());
    const int64_t ne = static_cast<int64_t>(hexahedron_elements.size());
    std::vector<uint32_t> conn(static_cast<size_t>(8 * ne));
    std::vector<double> bt(static_cast<size_t>(24 * ne));
    for (int64_t e = 0; e < ne; ++e) {
        const auto& vi = hexahedron_elements[e].get_verticesIndex();
        for (int k = 0; k < 8; ++k) {
            conn[8 * e + k] = static_cast<uint32_t>(vi[k]);
            for (int c = 0; c < 3; ++c) bt[24 * e + 3 * k + c] = all_BT[e](k, c);
        }
    }
    std::vector<double> x0(static_cast<size_t>(3 * nn));
    for (int64_t n = 0; n < nn; ++n)
        for (int c = 0; c < 3; ++c) x0[3 * n + c] = vertices[n][c];
    ensc_mesh_desc m{};
    m.n_nodes = nn;
    m.n_elements = ne;
    m.conn = conn.data();
    m.x0 = x0.data();
    m.v0 = solution_v.data();
    m.bt = bt.data();
    m.vol0 = all_Volume.data();
    m.inv_mass = inv_mass_matrix.data();
    ensc_material mat{};
    mat.E = mMatElastic.E;
    mat.nu = mMatElastic.v;
    mat.rho = mMatElastic.rho;
    mat.yield_stress = opt_.yield_stress;
    mat.hardening_modulus = opt_.hardening_modulus;
    ensc_params p{};
    p.c_dr = c_dr;
    p.c_cr = c_cr;
    p.factor_timestep = factor_timeStep;
    p.cvisl = Cvisl;
    p.cvisq = Cvisq;
    p.total_time = totalTime;
    p.precision = opt_.precision;
    p.device = opt_.device;
    p.stream = nullptr;
    p.graph_chunk = opt_.graph_chunk;
    if (h_) {
        ensc_destroy(h_);
        h_ = nullptr;
    }
    const int rc = ensc_create(&m, &mat, &p, &h_);
    if (rc != ENSC_OK) {
        h_ = nullptr;
        throw std::runtime_error("ensc_create failed (" + std::to_string(rc) + "): " + ensc_last_error(nullptr));
    }
}

namespace {

// Per-DOF codes of the current step's conditions, resolved as
// apply_boundary_condition_vec / apply_boundary_condition_a resolve them
// (exDyna3D.cpp:379-490, 2029-2145): velocity conditions by set or '#'-node
// name over a DOF range, then fixed DOFs of SPCs whose condition field is 1.
void resolve_conditions(const BoundaryCondition& bc, const std::map<std::string, std::vector<std::size_t>>& sets,
                        std::size_t n_nodes, std::vector<int8_t>& code, std::vector<double>& value) {
    code.assign(3 * n_nodes, 0);
    value.assign(3 * n_nodes, 0.0);
    std::vector<std::size_t> one;
    auto nodes = [&](const std::string& name) -> const std::vector<std::size_t>* {
        if (!name.empty() && name[0] == '#') {
            one.clear();
            try {
                one.push_back(static_cast<std::size_t>(std::stoi(name.substr(1)) - 1));
            } catch (...) {
            }
            return &one;
        }
        auto it = sets.find(name);
        return it == sets.end() ? nullptr : &it->second;
    };
    for (const auto& vb : bc.vel_nodes) {
        const auto* ids = nodes(vb.first);
        if (!ids) continue;
        for (std::size_t n : *ids) {
            if (n >= n_nodes) continue;
            for (std::size_t d = vb.second.first[0]; d <= vb.second.first[1] && d < 3; ++d) {
                code[3 * n + d] |= ENSC_BC_VELOCITY;
                value[3 * n + d] = vb.second.second;
            }
        }
    }
    for (const auto& sb : bc.spc_nodes) {
        if (sb.second[2] != 1) continue;
        const auto* ids = nodes(sb.first);
        if (!ids) continue;
        for (std::size_t n : *ids) {
            if (n >= n_nodes) continue;
            for (std::size_t d = sb.second[0]; d <= sb.second[1] && d < 3; ++d) code[3 * n + d] |= ENSC_BC_FIXED;
        }
    }
}

}  // namespace

// The conditions and gravity load setCurrentStep has made current, on the
// device.  ensc_set_bcs also applies the velocity conditions to the device
// velocities, as setCurrentStep does on the host (:1911).
void exDyna3D_GPU::upload_step_conditions() {
    std::vector<int8_t> code;
    std::vector<double> value;
    resolve_conditions(currentBoundary, map_set_node_list, vertices.size(), code, value);
    check(ensc_set_bcs(h_, code.data(), value.data()), "ensc_set_bcs");
    const auto& g = steps[currentStepIndex].gravity;
    if (std::get<0>(g)) {
        const double dir[3] = {std::get<3>(g), std::get<4>(g), std::get<5>(g)};
        check(ensc_set_gravity(h_, 1, std::get<2>(g), dir), "ensc_set_gravity");
        // a named amplitude that the deck never defines leaves the factor at
        // 1 (the reference reads past an empty table there)
        std::vector<double> pairs;
        const std::string& name = std::get<1>(g);
        if (!name.empty()) {
            auto it = map_amp_list.find(name);
            if (it != map_amp_list.end())
                for (const auto& pt : it->second) {
                    pairs.push_back(pt[0]);
                    pairs.push_back(pt[1]);
                }
        }
        check(ensc_set_gravity_amplitude(h_, static_cast<int32_t>(pairs.size() / 2),
                                         pairs.empty() ? nullptr : pairs.data()),
              "ensc_set_gravity_amplitude");
    } else {
        const double zero[3] = {0.0, 0.0, 0.0};
        check(ensc_set_gravity(h_, 0, 0.0, zero), "ensc_set_gravity");
        check(ensc_set_gravity_amplitude(h_, 0, nullptr), "ensc_set_gravity_amplitude");
    }
}

// Device state into the reference's arrays.
void exDyna3D_GPU::download_state() {
    const std::size_t nn = vertices.size();
    std::vector<double> x(3 * nn);
    static_assert(sizeof(std::array<double, 6>) == 6 * sizeof(double), "sigma rows must be packed");
    static_assert(sizeof(std::array<double, 12>) == 12 * sizeof(double), "QIA rows must be packed");
    check(ensc_download(h_, x.data(), solution_u.data(), solution_v.data(),
                        reinterpret_cast<double*>(all_sigma.data()), reinterpret_cast<double*>(all_QIA.data()),
                        nullptr),
          "ensc_download");
    for (std::size_t n = 0; n < nn; ++n)
        for (int c = 0; c < 3; ++c) vertices[n][c] = x[3 * n + c];
    check(ensc_download_reactions(h_, solution_rf.data()), "ensc_download_reactions");
}

// F = I + u_e B0^T per element (compute_deformation_gradient,
// exDyna3D.cpp:862-866), for the strain measure output_results writes.
void exDyna3D_GPU::update_strain_measure() {
    const std::size_t ne = hexahedron_elements.size();
    if (all_F.size() != ne) return;
    for (std::size_t e = 0; e < ne; ++e) {
        const auto& vi = hexahedron_elements[e].get_verticesIndex();
        Eigen::Matrix<Types::Real, 3, 3> F = Eigen::Matrix<Types::Real, 3, 3>::Identity();
        for (int k = 0; k < 8; ++k)
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) F(r, c) += solution_u[3 * vi[k] + r] * all_BT[e](k, c);
        all_F[e] = F;
    }
}

// The fields of a snapshot into the reference's arrays, then the
// reference's own output_results() (exDyna3D.cpp:207-336) at the snapshot's
// time.
void exDyna3D_GPU::write_snapshot(const ensc_snapshot& sn) {
    const std::size_t nn = vertices.size(), ne = hexahedron_elements.size();
    for (std::size_t n = 0; n < nn; ++n)
        for (int c = 0; c < 3; ++c) vertices[n][c] = sn.x[3 * n + c];
    std::copy(sn.u, sn.u + 3 * nn, solution_u.data());
    std::copy(sn.v, sn.v + 3 * nn, solution_v.data());
    std::copy(sn.a, sn.a + 3 * nn, solution_a.data());
    std::copy(sn.rf, sn.rf + 3 * nn, solution_rf.data());
    std::copy(sn.sigma, sn.sigma + 6 * ne, reinterpret_cast<double*>(all_sigma.data()));
    const Types::Real t = time, d0 = dt_i, d1 = dt_i_1;
    time = sn.time;
    dt_i = sn.dt_i;
    dt_i_1 = sn.dt_i_1;
    update_strain_measure();
    output_results();
    time = t;
    dt_i = d0;
    dt_i_1 = d1;
}

void exDyna3D_GPU::take_report(const ensc_step_report& r) {
    time = r.time;
    dt_i = r.dt_i;
    dt_i_1 = r.dt_i_1;
    cycles_ += r.cycles;
}

void exDyna3D_GPU::run() {
    // exDyna3D::run()'s prologue (exDyna3D.cpp:55-67), on the host as there
    init();
    mMatElastic.update();
    calculate_time_interval();
    get_fsiSph_virtualParticles_and_vel(0, 1.0 / 10.0);
    create_device();
    if (solution_a.size() != static_cast<Eigen::Index>(3 * vertices.size())) solution_a.resize(3 * vertices.size());
    for (std::size_t s = 1; s < steps.size(); ++s) {
        if (s > 1) download_state();  // the step switch acts on the current state
        setCurrentStep(s);
        upload_step_conditions();
        const Types::Real stepEnd = time + steps[s].timePeriod;
        bool run_cycles = true;
        while (time < stepEnd && time < totalTime) {
            if (run_cycles) {
                int64_t max_cycles = kCycleBound;
                double pause = HUGE_VAL;
                if (opt_.write_output) {
                    // output is due in the cycle in which time reaches time_output;
                    // when it is due already, that is the next cycle
                    if (!(time < time_output))
                        max_cycles = 1;
                    else
                        pause = time_output;
                }
                ensc_step_report r{};
                const int rc = ensc_step_until(h_, max_cycles, stepEnd, pause, &r);
                take_report(r);
                check(rc, "ensc_step_until");
                if (r.cycles == 0) break;
            }
            run_cycles = true;
            if (opt_.write_output && (time >= time_output || time >= totalTime)) {
                // capture the fields on the device, let the cycles up to the
                // next output time run while the copy and the file writing
                // proceed on the host, then take their report
                check(ensc_snapshot_begin(h_), "ensc_snapshot_begin");
                const Types::Real next = time_output + time_interval;  // output_results advances it so
                bool ahead = false;
                if (time < stepEnd && time < totalTime && next > time && dt_i > 0.0) {
                    const double span = std::min<double>(next, stepEnd) - time;
                    const double est = std::ceil(span / dt_i * 1.02) + 2.0;
                    const int64_t n = static_cast<int64_t>(std::min(est, static_cast<double>(kAheadCycles)));
                    check(ensc_step_until_async(h_, n, stepEnd, next), "ensc_step_until_async");
                    ahead = true;
                }
                ensc_snapshot sn{};
                check(ensc_snapshot_wait(h_, &sn), "ensc_snapshot_wait");
                write_snapshot(sn);
                if (ahead) {
                    ensc_step_report r{};
                    const int rc = ensc_sync(h_, &r);
                    take_report(r);
                    check(rc, "ensc_sync");
                    // the cycles ran up to the next output time: that output
                    // is due now, before any further cycle
                    run_cycles = !(time >= time_output || time >= totalTime);
                }
            }
        }
    }
    download_state();
}

namespace {

struct Record {
    std::string bytes;
    template <typename T>
    void pod(const T& v) {
        bytes.append(reinterpret_cast<const char*>(&v), sizeof(T));
    }
    void str(const std::string& s) {
        pod(static_cast<uint64_t>(s.size()));
        bytes.append(s);
    }
    void sizes(const std::vector<std::size_t>& v) {
        pod(static_cast<uint64_t>(v.size()));
        for (std::size_t x : v) pod(static_cast<uint64_t>(x));
    }
};

}  // namespace

std::string exDyna3D_GPU::model_record() {
    Record r;
    r.pod(static_cast<uint64_t>(vertices.size()));
    for (const auto& x : vertices) r.pod(x);
    r.pod(static_cast<uint64_t>(hexahedron_elements.size()));
    for (auto& el : hexahedron_elements) {
        r.pod(el.get_PID());
        r.pod(el.get_MID());
        const auto& vi = el.get_verticesIndex();
        r.pod(static_cast<uint64_t>(vi.size()));
        for (auto v : vi) r.pod(v);
    }
    for (const auto* sets : {&map_set_node_list, &map_set_ele_list}) {
        r.pod(static_cast<uint64_t>(sets->size()));
        for (const auto& s : *sets) {
            r.str(s.first);
            r.sizes(s.second);
        }
    }
    r.pod(static_cast<uint64_t>(map_set_surface_list.size()));
    for (const auto& s : map_set_surface_list) {
        r.str(s.first);
        r.str(s.second.first);
        r.str(s.second.second);
    }
    r.pod(static_cast<uint64_t>(steps.size()));
    for (const auto& st : steps) {
        r.str(st.name);
        r.pod(st.timePeriod);
        r.pod(st.resetSpcBoundary);
        r.pod(st.resetVelBoundary);
        r.pod(st.resetDload);
        r.pod(st.resetDsload);
        r.pod(static_cast<uint64_t>(st.boundary.spc_nodes.size()));
        for (const auto& b : st.boundary.spc_nodes) {
            r.str(b.first);
            for (auto v : b.second) r.pod(static_cast<uint64_t>(v));
        }
        r.pod(static_cast<uint64_t>(st.boundary.vel_nodes.size()));
        for (const auto& b : st.boundary.vel_nodes) {
            r.str(b.first);
            for (auto v : b.second.first) r.pod(static_cast<uint64_t>(v));
            r.pod(b.second.second);
        }
        r.pod(std::get<0>(st.gravity));
        if (std::get<0>(st.gravity)) {  // the other fields are set only with gravity on
            r.str(std::get<1>(st.gravity));
            r.pod(std::get<2>(st.gravity));
            r.pod(std::get<3>(st.gravity));
            r.pod(std::get<4>(st.gravity));
            r.pod(std::get<5>(st.gravity));
        }
        r.pod(static_cast<uint64_t>(st.dsload.size()));
        for (const auto& d : st.dsload) {
            r.str(std::get<0>(d));
            r.str(std::get<1>(d));
            r.str(std::get<2>(d));
            r.pod(std::get<3>(d));
        }
    }
    r.pod(static_cast<uint64_t>(ini_vel_generation.size()));
    for (const auto& iv : ini_vel_generation) {
        r.str(iv.first);
        r.pod(static_cast<uint64_t>(iv.second.first));
        r.pod(iv.second.second);
    }
    r.pod(static_cast<uint64_t>(map_amp_list.size()));
    for (const auto& a : map_amp_list) {
        r.str(a.first);
        r.pod(static_cast<uint64_t>(a.second.size()));
        for (const auto& pt : a.second) r.pod(pt);
    }
    for (double v : {mMatElastic.E, mMatElastic.rho, mMatElastic.v, mMatElastic.G, mMatElastic.K, mMatElastic.lambda,
                     mMatElastic.WOS, Cvisl, Cvisq, totalTime, time_interval})
        r.pod(v);
    r.pod(time_interval_set);
    return r.bytes;
}

void exDyna3D_GPU::dump_state(const std::string& path) const {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    const int64_t nn = static_cast<int64_t>(vertices.size());
    const int64_t ne = static_cast<int64_t>(hexahedron_elements.size());
    const int64_t cyc = cycles_;
    std::fwrite("ENSCDMP1", 1, 8, f);
    std::fwrite(&nn, 8, 1, f);
    std::fwrite(&ne, 8, 1, f);
    std::fwrite(&cyc, 8, 1, f);
    const double scal[16] = {time,           dt_i,          dt_i_1,        totalTime,
                             mMatElastic.E,  mMatElastic.v, mMatElastic.rho, mMatElastic.G,
                             mMatElastic.K,  mMatElastic.lambda, mMatElastic.WOS, c_dr,
                             c_cr,           factor_timeStep, Cvisl,       Cvisq};
    std::fwrite(scal, 8, 16, f);
    std::vector<double> buf(static_cast<size_t>(3 * nn));
    for (int64_t n = 0; n < nn; ++n)
        for (int c = 0; c < 3; ++c) buf[3 * n + c] = vertices[n][c];
    std::fwrite(buf.data(), 8, buf.size(), f);
    std::fwrite(solution_u.data(), 8, 3 * nn, f);
    std::fwrite(solution_v.data(), 8, 3 * nn, f);
    std::fwrite(inv_mass_matrix.data(), 8, 3 * nn, f);
    std::fwrite(solution_rf.data(), 8, 3 * nn, f);
    std::fwrite(all_sigma.data(), 8, 6 * ne, f);
    std::fwrite(all_QIA.data(), 8, 12 * ne, f);
    buf.assign(static_cast<size_t>(24 * ne), 0.0);
    for (int64_t e = 0; e < ne; ++e)
        for (int k = 0; k < 8; ++k)
            for (int c = 0; c < 3; ++c) buf[24 * e + 3 * k + c] = all_BT[e](k, c);
    std::fwrite(buf.data(), 8, buf.size(), f);
    std::fwrite(all_Volume.data(), 8, ne, f);
    std::fwrite(dtStable.data(), 8, ne, f);
    std::fwrite(all_Length.data(), 8, ne, f);
    std::vector<uint32_t> conn(static_cast<size_t>(8 * ne));
    for (int64_t e = 0; e < ne; ++e) {
        const auto& vi = hexahedron_elements[e].get_verticesIndex();
        for (int k = 0; k < 8; ++k) conn[8 * e + k] = static_cast<uint32_t>(vi[k]);
    }
    std::fwrite(conn.data(), 4, conn.size(), f);
    std::vector<int8_t> code;
    std::vector<double> value;
    resolve_conditions(currentBoundary, map_set_node_list, vertices.size(), code, value);
    std::fwrite(code.data(), 1, code.size(), f);
    std::fwrite(value.data(), 8, value.size(), f);
    std::fclose(f);
}

}  // namespace EnSC
