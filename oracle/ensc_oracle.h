/* Test infrastructure -- NOT part of the product.
 *
 * Plain-C restatement of the EnSCDynamics explicit central-difference stepper
 * (reference: Explicit3D/source/exDyna3D.cpp), used by tests/ and by
 * bench.py's CPU-baseline leg as the checker.  The product (the CUDA stepper
 * behind include/ensc_gpu.h) never links or calls this code.
 *
 * Arrays follow the reference's own layouts: nodal vectors interleaved xyz
 * (solution_u/v, exDyna3D.h:159-167), vertices AoS (exDyna3D.h:141), sigma
 * [xx,yy,zz,xy,xz,yz] (exDyna3D.h:146), QIA[12] (exDyna3D.h:148), B0^T as a
 * row-major 8x3 per element (all_BT, exDyna3D.h:154), connectivity 8 x uint32
 * per element (ElementBase.h:110).
 *
 * Parity status: pinned against the compiled reference stepper (oracle/_ref)
 * by tests/test_oracle_vs_reference.py; the reference evaluates some 3x8*8x3
 * Eigen products in an alignment-dependent order, so agreement is to
 * round-off (documented tolerance), not bit-for-bit.  The J2 return mapping
 * and the energy sums have no reference counterpart; they are pinned by
 * known-answer tests and by reducing bit-exactly to the elastic path when the
 * yield stress is disabled.
 */
#ifndef ENSC_ORACLE_H
#define ENSC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* material (Material_elastic.h:8-21, Material_elastic.cpp:9-14) */
    double E, nu, rho;
    double G, K, lambda, wos;      /* filled by ensc_oracle_material_update */
    double yield0;                 /* J2 initial yield stress; <= 0 -> elastic */
    double hardening;              /* J2 linear isotropic hardening modulus H */
    /* solver controls (exDyna3D.h:176-185, read_project_txt exDyna3D.cpp:698) */
    double c_dr, c_cr, factor, cvisl, cvisq;
    double total_time;
    /* gravity (StepData::gravity, apply_gravity exDyna3D.cpp:800-826) with
     * an optional amplitude table (map_amp_list, read by DataIn::AMP
     * dataIn.cpp:1244-1270): amp_n (time, value) pairs, none when amp_n = 0 */
    int32_t gravity_on;
    double gravity_value, gravity_dir[3];
    int32_t amp_n;
    const double* amp;
} ensc_oracle_params;

typedef struct {
    int64_t nn, ne;
    const uint32_t* conn;          /* ne*8 */
    double* x;                     /* nn*3 current coordinates */
    double* u;                     /* nn*3 */
    double* v;                     /* nn*3 */
    double* inv_mass;              /* nn*3 */
    double* rf;                    /* nn*3 reactions */
    double* sigma;                 /* ne*6 */
    double* qia;                   /* ne*12 */
    double* eps_p;                 /* ne (J2 equivalent plastic strain) */
    const double* bt;              /* ne*24 */
    const double* vol0;            /* ne */
    const double* cbrt_v0;         /* ne: cbrt(V0) */
    const double* cbrt_v0sq;       /* ne: cbrt(V0*V0) */
    double* len;                   /* ne scratch: min edge */
    double* dtstable;              /* ne scratch: element dt */
    double* force;                 /* nn*3 scratch: assembled force */
    double* slots;                 /* 8*nn*3 scratch: per-local-slot vectors */
    const int8_t* bc_code;         /* nn*3: bit0 fixed, bit1 velocity */
    const double* bc_value;        /* nn*3 */
    double time, dt_i, dt_i_1;
    int64_t cycles;
    /* energy sums: [0] kinetic, [1] internal (stress work), [2] hourglass,
       [3] bulk viscosity, [4] external work (gravity + reactions) */
    double energy[5];
} ensc_oracle_state;

void ensc_oracle_material_update(ensc_oracle_params* p);

/* exDyna3D::deal_amp (exDyna3D.cpp:1222-1278): the amplitude factor applied
 * to gravity in a cycle at `time` with step dt, from n (time, value) pairs. */
double ensc_oracle_amplitude(const double* amp, int32_t n, double time, double dt);

/* compute_invMassMatrix (exDyna3D.cpp:492-515) with FEValues::reinit at the
 * single Gauss point (fevalues.h:232-265): B0^T, V0 and the inverse lumped
 * mass; also cbrt(V0) and cbrt(V0^2) used by the element kernel. */
void ensc_oracle_setup(int64_t nn, int64_t ne, const uint32_t* conn, const double* x0, double rho,
                       double* bt, double* vol0, double* cbrt_v0, double* cbrt_v0sq,
                       double* inv_mass);

/* cbrt(V0) and cbrt(V0^2) with the C library, as the reference's std::cbrt
 * (exDyna3D.cpp:1040, 1081). */
void ensc_oracle_cbrt_pair(int64_t ne, const double* vol0, double* cbrt_v0, double* cbrt_v0sq);

/* The force pass that exDyna3D::init() runs with dt = 0 and no boundary
 * conditions (exDyna3D.cpp:126-141): fills len[] and dtstable[]. */
void ensc_oracle_init_pass(const ensc_oracle_params* p, ensc_oracle_state* s);

/* apply_boundary_condition_vec (exDyna3D.cpp:379-490). */
void ensc_oracle_apply_bc_v(ensc_oracle_state* s);

/* Kinetic energy of the current velocity field. */
double ensc_oracle_kinetic(const ensc_oracle_state* s);

/* Runs cycles of the run() loop body (exDyna3D.cpp:86-100) while
 * time < step_end, at most max_cycles; returns the number of cycles run. */
int64_t ensc_oracle_cycles(const ensc_oracle_params* p, ensc_oracle_state* s,
                           int64_t max_cycles, double step_end);

#ifdef __cplusplus
}
#endif

#endif
