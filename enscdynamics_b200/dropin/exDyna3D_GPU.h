// exDyna3D_GPU: the reference solver class with its time-step loop on the GPU.
//
// A drop-in for EnSC::exDyna3D (Explicit3D/include/exDyna3D.h:36): the deck
// is read by the reference's own DataIn (a friend of exDyna3D that fills the
// subclass unchanged, dataIn.h:35), init() is the reference's own -- project
// controls, element constants, lumped mass, initial conditions -- and so are
// the step switches (setCurrentStep, exDyna3D.cpp:1760-1940, with their
// boundary-condition and gravity inheritance) and the result output
// (output_results, :207-336).  Only run() is overridden (exDyna3D.h:46): the
// cycles of each step -- stable dt, last-step clamp and computeSate
// (:86-100) -- run on the device through the ensc_* C ABI
// (include/ensc_gpu.h), and the state comes back into the reference's own
// arrays (vertices, solution_u, solution_v, solution_rf, all_sigma, all_QIA,
// time, dt_i, dt_i_1) at every output time and step end.
//
// Output: at an output time the fields are captured on the device
// (ensc_snapshot_begin) and the cycles up to the next output time are
// enqueued (ensc_step_until_async) before the host copies and writes them,
// so the file writing overlaps the stepping.
//
// Differences from exDyna3D::run():
//   * results are written after the cycle in which time reaches the next
//     output time; the reference writes them from inside that cycle, before
//     its velocity update (computeSate :788), so the written velocities and
//     positions are those at the end of the same cycle (the acceleration is
//     that cycle's, as the reference writes it);
//   * the strain field is recomputed on the host from u; the nodal-force
//     field is zero, as the reference's own solution_f, which it never fills
//     (exDyna3D.cpp:157,179);
//   * FSI virtual-particle forces are not applied (none exist unless a
//     coupled SPH solver provides them);
//   * a step whose end lies beyond totalTime ends at totalTime (the reference
//     would keep cycling with time clamped to totalTime).
#pragma once

#include "ensc_gpu.h"
#include "exDyna3D.h"

#include <cstdint>
#include <string>

namespace EnSC {

class exDyna3D_GPU : public exDyna3D {
    friend class DataInFast;  // the fast deck reader fills the model as DataIn does

public:
    struct Options {
        int32_t precision = ENSC_FP64;   // ENSC_FP64 or ENSC_MIXED
        int32_t device = 0;              // CUDA device ordinal
        int32_t graph_chunk = 0;         // cycles per captured graph (0: default)
        bool write_output = true;        // output_results() at the reference's output times
        // J2 plasticity (the reference material is hypoelastic; yield <= 0
        // keeps it so)
        double yield_stress = 0.0;
        double hardening_modulus = 0.0;
    };

    exDyna3D_GPU();
    explicit exDyna3D_GPU(const Options& options);
    ~exDyna3D_GPU();
    exDyna3D_GPU(const exDyna3D_GPU&) = delete;
    exDyna3D_GPU& operator=(const exDyna3D_GPU&) = delete;

    // exDyna3D::run() with the cycles on the GPU.  Throws std::runtime_error
    // with the library's message when a call fails or the solution becomes
    // non-finite or inverts an element.
    void run() override;

    int64_t cycles() const { return cycles_; }
    std::size_t n_vertices() const { return vertices.size(); }
    std::size_t n_elements() const { return hexahedron_elements.size(); }

    // Everything a deck reader fills in the solver (nodes, elements, sets,
    // surfaces, steps with their conditions and loads, initial velocities,
    // amplitudes, material, bulk viscosity, total time, output interval) as
    // one byte string, for comparing two readers on the same deck.
    std::string model_record();

    // Writes the solver state in the ENSCDMP1 layout (counts, clock and
    // controls, then x, u, v, inverse mass, reactions, sigma, QIA, B0^T, V0,
    // element dt, min edge, connectivity, per-DOF BC codes and values).
    void dump_state(const std::string& path) const;

protected:
    void create_device();
    void upload_step_conditions();
    void download_state();
    void update_strain_measure();
    void write_snapshot(const ensc_snapshot& sn);
    void take_report(const ensc_step_report& r);
    void check(int rc, const char* what) const;

    Options opt_;
    ensc_handle* h_ = nullptr;
    int64_t cycles_ = 0;
};

}  // namespace EnSC
