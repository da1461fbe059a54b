// ensc_reader_bench: reads a deck with the reference reader (DataIn,
// Explicit3D/source/dataIn.cpp) and with DataInFast, times both, and checks
// that they fill the solver identically (every member a reader sets,
// compared byte for byte).
//
//   ensc_reader_bench deck.inp [repeats]
//
// Prints one JSON line: nodes, elements, best-of-repeats seconds of each
// reader, and "identical".
#include "dataIn.h"
#include "deck_reader.h"
#include "exDyna3D_GPU.h"
#include "spdlog/spdlog.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace {
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s deck.inp [repeats]\n", argv[0]);
        return 2;
    }
    spdlog::set_level(spdlog::level::err);
    const std::string deck = argv[1];
    const int repeats = argc > 2 ? std::max(1, std::atoi(argv[2])) : 1;
    double t_ref = 1e30, t_fast = 1e30;
    std::string rec_ref, rec_fast;
    std::size_t nn = 0, ne = 0;
    try {
        for (int i = 0; i < repeats; ++i) {
            EnSC::exDyna3D_GPU a;
            const double t0 = now_s();
            EnSC::DataIn(a).read_inp(deck);
            t_ref = std::min(t_ref, now_s() - t0);
            if (i == 0) rec_ref = a.model_record();
        }
        for (int i = 0; i < repeats; ++i) {
            EnSC::exDyna3D_GPU b;
            const double t0 = now_s();
            EnSC::DataInFast(b).read_inp(deck);
            t_fast = std::min(t_fast, now_s() - t0);
            if (i == 0) {
                rec_fast = b.model_record();
                nn = b.n_vertices();
                ne = b.n_elements();
            }
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ensc_reader_bench: %s\n", e.what());
        return 1;
    }
    std::printf("{\"deck\": \"%s\", \"nodes\": %zu, \"elements\": %zu, \"reference_s\": %.6f, \"fast_s\": %.6f, "
                "\"speedup\": %.3f, \"identical\": %s, \"record_bytes\": %zu}\n",
                deck.c_str(), nn, ne, t_ref, t_fast, t_ref / t_fast, rec_ref == rec_fast ? "true" : "false",
                rec_fast.size());
    return rec_ref == rec_fast ? 0 : 3;
}
