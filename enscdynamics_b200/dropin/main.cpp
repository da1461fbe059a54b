// ensc_dropin: the reference program (main.cpp of the reference) with
// exDyna3D_GPU in place of exDyna3D.
//
// As the reference, run it from a directory holding project.txt; without a
// deck argument it solves inp/<first non-comment line of project.txt>.
//
//   ensc_dropin [--precision fp64|mixed] [--device N] [--graph-chunk N]
//               [--yield S --hardening H] [--no-output] [--dump FILE]
//               [--reference-reader] [--log-level LEVEL] [deck.inp]
//
// The deck is read with DataInFast (deck_reader.h), which fills the solver
// as the reference's DataIn does; --reference-reader uses DataIn itself.
//
// On success it prints one JSON line: cycles run, final time, dt, and the
// wall time of run().
#include "dataIn.h"
#include "deck_reader.h"
#include "exDyna3D_GPU.h"
#include "spdlog/spdlog.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

namespace {

std::string deck_from_project() {
    std::ifstream fin("project.txt");
    if (!fin.is_open()) return "";
    std::string line;
    while (std::getline(fin, line)) {
        if (line.empty() || line[0] == '#') continue;
        return "inp/" + line;
    }
    return "";
}

int usage(const char* argv0) {
    std::fprintf(stderr,
                 "usage: %s [--precision fp64|mixed] [--device N] [--graph-chunk N] [--yield S --hardening H] "
                 "[--no-output] [--dump FILE] [--reference-reader] [--log-level LEVEL] [deck.inp]\n",
                 argv0);
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    EnSC::exDyna3D_GPU::Options opt;
    std::string deck, dump;
    std::string level = "warn";
    bool reference_reader = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> const char* { return i + 1 < argc ? argv[++i] : nullptr; };
        const char* v = nullptr;
        if (a == "--precision" && (v = next())) {
            if (!std::strcmp(v, "fp64")) opt.precision = ENSC_FP64;
            else if (!std::strcmp(v, "mixed")) opt.precision = ENSC_MIXED;
            else return usage(argv[0]);
        } else if (a == "--device" && (v = next())) {
            opt.device = std::atoi(v);
        } else if (a == "--graph-chunk" && (v = next())) {
            opt.graph_chunk = std::atoi(v);
        } else if (a == "--yield" && (v = next())) {
            opt.yield_stress = std::atof(v);
        } else if (a == "--hardening" && (v = next())) {
            opt.hardening_modulus = std::atof(v);
        } else if (a == "--reference-reader") {
            reference_reader = true;
        } else if (a == "--no-output") {
            opt.write_output = false;
        } else if (a == "--dump" && (v = next())) {
            dump = v;
        } else if (a == "--log-level" && (v = next())) {
            level = v;
        } else if (!a.empty() && a[0] != '-' && deck.empty()) {
            deck = a;
        } else {
            return usage(argv[0]);
        }
    }
    spdlog::set_level(spdlog::level::from_str(level));
    if (deck.empty()) deck = deck_from_project();
    if (deck.empty()) {
        std::fprintf(stderr, "no deck: give one or write its name in project.txt\n");
        return 2;
    }
    try {
        EnSC::exDyna3D_GPU solver(opt);
        const auto tr = std::chrono::steady_clock::now();
        if (reference_reader) EnSC::DataIn(solver).read_inp(deck);
        else EnSC::DataInFast(solver).read_inp(deck);
        const double read_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - tr).count();
        const auto t0 = std::chrono::steady_clock::now();
        solver.run();
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (!dump.empty()) solver.dump_state(dump);
        std::printf("{\"cycles\": %lld, \"read_s\": %.6f, \"run_s\": %.6f}\n", static_cast<long long>(solver.cycles()),
                    read_s, secs);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ensc_dropin: %s\n", e.what());
        return 1;
    }
    return 0;
}
