// Test infrastructure: harness around the reference CPU stepper.
//
// This file is compiled together with the UNMODIFIED reference sources
// (Explicit3D/source/{exDyna3D,dataIn,Element_HexN8,Material_elastic,
// gauss_integral_1d}.cpp) by oracle/Makefile; the result lands in oracle/_ref/
// and is used only by the tests and by bench.py's CPU-baseline leg, as the
// checker and the reference timing -- never as the product.
//
// It subclasses EnSC::exDyna3D (Explicit3D/include/exDyna3D.h:36), whose
// state is protected and whose run()/computeSate() are virtual
// (exDyna3D.h:46,75), to
//   * run a bounded number of central-difference cycles with the same loop as
//     exDyna3D::run() (Explicit3D/source/exDyna3D.cpp:77-101),
//   * or call exDyna3D::run() itself,
//   * and dump the solver state (u, v, x, sigma, QIA, mass, B0^T, V0, ...) as
//     raw little-endian doubles so the GPU stepper can be compared with it.
//
// Usage (run from the directory that holds project.txt, as the reference
// requires, exDyna3D.cpp:705):
//   ensc_ref_harness <deck.inp> cycles <N> <dump.bin>
//   ensc_ref_harness <deck.inp> full <dump.bin>
//   ensc_ref_harness <deck.inp> setup <dump.bin>  (state after init() and
//       setCurrentStep(1); the u field carries the velocities init() left,
//       before the first step's boundary conditions)
//   ensc_ref_harness <deck.inp> time <N>          (timing JSON on stdout)
// OMP_NUM_THREADS selects the OpenMP thread count as for the reference.
#include "exDyna3D.h"
#include "dataIn.h"
#include "spdlog/spdlog.h"

#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

class RefHarness : public EnSC::exDyna3D {
public:
    long cycles_done = 0;
    long cycle_cap = -1;  // < 0: unbounded
    std::vector<double> v_read;  // setup dumps: written in place of u (keep_velocity)

    // Counts cycles; the body of a cycle is the reference's own computeSate().
    void computeSate() override {
        ++cycles_done;
        EnSC::exDyna3D::computeSate();
    }

    // Everything exDyna3D::run() does before its step loop
    // (exDyna3D.cpp:55-67), without the debug prints.
    void prologue() {
        init();
        mMatElastic.update();
        calculate_time_interval();
        get_fsiSph_virtualParticles_and_vel(0, 1.0 / 10.0);
    }

    // The step loop of exDyna3D::run() (exDyna3D.cpp:77-101), stopped after
    // cycle_cap cycles when cycle_cap >= 0.
    void step_loop() {
        for (std::size_t s = 1; s < steps.size(); ++s) {
            if (cycle_cap >= 0 && cycles_done >= cycle_cap) return;
            setCurrentStep(s);
            const double stepEnd = time + steps[s].timePeriod;
            while (time < stepEnd) {
                if (cycle_cap >= 0 && cycles_done >= cycle_cap) return;
                update_minVertex_perMaterial_and_dt();
                if (time + dt_i_1 > stepEnd) {
                    const double remaining = stepEnd - time;
                    dt_i = dt_i_1 = remaining;
                }
                computeSate();
            }
        }
    }

    void full_run() { EnSC::exDyna3D::run(); }

    // The velocities init() left (the deck's initial conditions, before the
    // first step's boundary conditions), for the setup dump.
    void keep_velocity() { v_read.assign(solution_v.data(), solution_v.data() + solution_v.size()); }

    std::size_t n_nodes() const { return vertices.size(); }
    std::size_t n_elements() const { return hexahedron_elements.size(); }

    // Per-DOF boundary-condition codes of the current step, resolved the way
    // apply_boundary_condition_vec / apply_boundary_condition_a resolve them
    // (exDyna3D.cpp:379-490, 2029-2145): bit 1 = velocity BC (value), bit 0 =
    // fixed (SPC with condition == 1).
    void bc_codes(std::vector<int8_t>& code, std::vector<double>& value) const {
        const std::size_t ndof = 3 * vertices.size();
        code.assign(ndof, 0);
        value.assign(ndof, 0.0);
        auto nodes_of = [&](const std::string& name, std::vector<std::size_t>& out) {
            out.clear();
            if (!name.empty() && name[0] == '#') {
                try { out.push_back(static_cast<std::size_t>(std::stoi(name.substr(1)) - 1)); } catch (...) {}
            } else {
                auto it = map_set_node_list.find(name);
                if (it != map_set_node_list.end()) out = it->second;
            }
        };
        std::vector<std::size_t> ids;
        for (const auto& vb : currentBoundary.vel_nodes) {
            nodes_of(vb.first, ids);
            for (std::size_t n : ids)
                for (std::size_t d = vb.second.first[0]; d <= vb.second.first[1]; ++d) {
                    code[3 * n + d] |= 2;
                    value[3 * n + d] = vb.second.second;
                }
        }
        for (const auto& sb : currentBoundary.spc_nodes) {
            nodes_of(sb.first, ids);
            if (sb.second[2] != 1) continue;
            for (std::size_t n : ids)
                for (std::size_t d = sb.second[0]; d <= sb.second[1]; ++d) code[3 * n + d] |= 1;
        }
    }

    void dump(const char* path) const {
        FILE* f = std::fopen(path, "wb");
        if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
        const int64_t nn = static_cast<int64_t>(vertices.size());
        const int64_t ne = static_cast<int64_t>(hexahedron_elements.size());
        const int64_t cyc = cycles_done;
        std::fwrite("ENSCDMP1", 1, 8, f);
        std::fwrite(&nn, 8, 1, f);
        std::fwrite(&ne, 8, 1, f);
        std::fwrite(&cyc, 8, 1, f);
        const double scal[16] = {time, dt_i, dt_i_1, totalTime,
                                 mMatElastic.E, mMatElastic.v, mMatElastic.rho, mMatElastic.G,
                                 mMatElastic.K, mMatElastic.lambda, mMatElastic.WOS, c_dr,
                                 c_cr, factor_timeStep, Cvisl, Cvisq};
        std::fwrite(scal, 8, 16, f);
        std::vector<double> buf;
        auto put = [&](const std::vector<double>& b) { std::fwrite(b.data(), 8, b.size(), f); };
        buf.resize(3 * nn);
        for (int64_t i = 0; i < nn; ++i)
            for (int c = 0; c < 3; ++c) buf[3 * i + c] = vertices[i][c];
        put(buf);                                                     // x
        for (int64_t i = 0; i < 3 * nn; ++i) buf[i] = v_read.empty() ? solution_u[i] : v_read[i];
        put(buf);                                                     // u (setup: v as read)
        for (int64_t i = 0; i < 3 * nn; ++i) buf[i] = solution_v[i];
        put(buf);                                                     // v
        for (int64_t i = 0; i < 3 * nn; ++i) buf[i] = inv_mass_matrix[i];
        put(buf);                                                     // inverse lumped mass
        for (int64_t i = 0; i < 3 * nn; ++i) buf[i] = solution_rf[i];
        put(buf);                                                     // reaction
        buf.resize(6 * ne);
        for (int64_t e = 0; e < ne; ++e)
            for (int c = 0; c < 6; ++c) buf[6 * e + c] = all_sigma[e][c];
        put(buf);                                                     // sigma
        buf.resize(12 * ne);
        for (int64_t e = 0; e < ne; ++e)
            for (int c = 0; c < 12; ++c) buf[12 * e + c] = all_QIA[e][c];
        put(buf);                                                     // QIA
        buf.resize(24 * ne);
        for (int64_t e = 0; e < ne; ++e)
            for (int i = 0; i < 8; ++i)
                for (int c = 0; c < 3; ++c) buf[24 * e + 3 * i + c] = all_BT[e](i, c);
        put(buf);                                                     // B0^T, row-major 8x3
        buf.resize(ne);
        for (int64_t e = 0; e < ne; ++e) buf[e] = all_Volume[e];
        put(buf);                                                     // V0
        for (int64_t e = 0; e < ne; ++e) buf[e] = dtStable[e];
        put(buf);                                                     // element dt
        for (int64_t e = 0; e < ne; ++e) buf[e] = all_Length[e];
        put(buf);                                                     // min edge
        std::vector<uint32_t> conn(8 * ne);
        for (int64_t e = 0; e < ne; ++e) {
            const auto& vi = hexahedron_elements[e].get_verticesIndex();
            for (int i = 0; i < 8; ++i) conn[8 * e + i] = vi[i];
        }
        std::fwrite(conn.data(), 4, conn.size(), f);                 // connectivity
        std::vector<int8_t> code;
        std::vector<double> value;
        bc_codes(code, value);
        std::fwrite(code.data(), 1, code.size(), f);                 // BC code per DOF
        put(value);                                                   // BC value per DOF
        std::fclose(f);
    }
};

double now_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr,
                     "usage: %s <deck.inp> cycles <N> <dump> | full <dump> | setup <dump> | time <N>\n",
                     argv[0]);
        return 2;
    }
    spdlog::set_level(spdlog::level::err);
    const std::string deck = argv[1];
    const std::string mode = argv[2];

    RefHarness h;
    EnSC::DataIn reader(h);
    const double t0 = now_s();
    reader.read_inp(deck);
    const double t1 = now_s();

    if (mode == "setup") {
        h.prologue();
        h.keep_velocity();
        h.setCurrentStep(1);
        h.dump(argv[3]);
        return 0;
    }
    if (mode == "full") {
        h.init();  // timed apart from the loop; run() skips its own init() afterwards
        const double t2 = now_s();
        h.full_run();
        const double t3 = now_s();
        h.dump(argv[3]);
        std::printf("{\"mode\": \"full\", \"cycles\": %ld, \"parse_s\": %.6f, \"loop_s\": %.6f}\n",
                    h.cycles_done, t1 - t0, t3 - t2);
        return 0;
    }
    if (mode == "cycles" || mode == "time") {
        h.cycle_cap = std::atol(argv[3]);
        h.prologue();
        const double t2 = now_s();
        h.step_loop();
        const double t3 = now_s();
        if (mode == "cycles") {
            if (argc < 5) { std::fprintf(stderr, "missing dump path\n"); return 2; }
            h.dump(argv[4]);
        }
        std::printf(
            "{\"mode\": \"%s\", \"cycles\": %ld, \"elements\": %zu, \"nodes\": %zu, \"threads\": %d, "
            "\"parse_s\": %.6f, \"loop_s\": %.6f}\n",
            mode.c_str(), h.cycles_done, h.n_elements(), h.n_nodes(),
            omp_get_max_threads(), t1 - t0, t3 - t2);
        return 0;
    }
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}
